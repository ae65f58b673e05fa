// Split-INT8 (Ozaki-style) block contraction on the tcgen05 INT8 tensor cores.
//
// Every operand block of a contraction is viewed as its GEMM matrix (A: M x K with
// the A-outer labels as rows, B: N x K with the B-outer labels as rows, K = the inner
// labels in A's order — the Ainter / Binter views of kernels::block_multiply,
// multiply.hpp:304-330, without materialising them in FP64).  Each row is scaled by
// a power of two 2^-e (e = exponent of the row's max |x|, per block) and cut into S
// balanced base-256 digits of the integer X = round(x * 2^(8S-1-e)), |X| <= 127 * 256^(S-1)
// (e is raised by one for the rare rows whose max lies within 1/128 below 2^e):
//     X = d_0 * 256^(S-1) + d_1 * 256^(S-2) + ... + d_(S-1),   every d_i in [-128, 127]
// (s8; zero-mean digits keep the dropped low-order products unbiased, so their error
// grows like sqrt(K) instead of K).  A * B is then the sum over digit pairs of
// exact INT8 x INT8 -> INT32 tensor-core products; pairs (i, j) with equal i + j share
// one power of two, so the S(S+1)/2 products with i + j <= S - 1 accumulate into S
// INT32 TMEM accumulators ("diagonals").  After each (A block, B block) task the
// diagonals are recombined in FP64, rescaled by 2^(e_row + e_col - 14 - 8d) and added
// to FP64 register accumulators; the output block is written once, in C's own label
// order, when the group's tasks are done.
//
// Truncation: each operand is exact to 2^-(8S-1) of its row maximum and the dropped
// pairs (i + j >= S) weigh at most ~S * 2^(2-8S) of row-max x col-max x K.  The slice
// count is chosen per task: the largest task of an output block gets the S the error
// target needs (S = 6, 21 INT8 products, for 1e-11), tasks 2^(8m) smaller get S - m,
// numerically zero blocks one digit.  This is the error-free splitting of Ozaki,
// Ogita, Oishi and Rump with the INT8 tensor-core digit layout of Ozaki / Uchino /
// Imamura's DGEMM emulation.
#include "tb_internal.hpp"
#include "tb_runtime.hpp"
#include "tb_sm100.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>

namespace tb {

void launch_contract_fp64(const Plan&, const WorkList&, double, double, int, const double*,
                          const double*, double*, cudaStream_t);

namespace {
using namespace sm100;

constexpr int MT = 128; // UMMA M: output rows of a tile
constexpr int KC = 32;  // bytes of K per pipeline stage (one INT8 MMA k-step)
constexpr int kMaxSmem = 227 * 1024; // dynamic shared memory per CTA on sm_100
constexpr int NEPI     = 256;           // epilogue threads of the default kernel (warps 2-9)
constexpr int NTHREADS = 64 + NEPI;     // warp 0 producer, warp 1 MMA issuer, warps 2-9 epilogue

// One operand block to split into digit slices.
struct SplitBlock {
  int64_t src_off; // element offset in the FP64 arena
  int64_t dst_off; // byte offset of the block's slices in the scratch
  int32_t exp_off; // first exponent (int32 per padded row)
  int32_t id;      // index into the per-block max-exponent array
  int32_t rows, K, rows_pad, K_pad, tile_rows;
  int32_t nr, nk, kcontig;
  int32_t rdim[kMaxClass], rstr[kMaxClass];
  int32_t kdim[kMaxClass], kstr[kMaxClass];
};

struct I8Task {
  int64_t a_off, b_off; // byte offsets of the A / B block slices
  int32_t a_exp, b_exp; // exponent index bases
  int32_t nkc;          // K_pad / KC
  int32_t pad;
};

struct I8TaskMeta {
  int32_t a_block, b_block; // max-exponent slots (B blocks after the A blocks)
  int32_t log2k;            // ceil(log2 K) of the task
};

struct I8Item {
  int32_t group, mt, nt, pad;
};

// One output tile as the producer hands it to the MMA issuer and the epilogue through a
// shared-memory queue slot: its item and group, and the row / column geometry of its C
// block (extents and strides of the row and column labels), worked out once per tile by
// the producer, off the consumers' critical path, and read by the epilogue threads from
// shared memory (indexing per-thread arrays by runtime label positions would put them
// in local memory).
struct TileRec {
  int64_t c_off;
  int32_t group, mt, nt, task_begin, task_end, M, N;
  int32_t mdim[kMaxClass], mstr[kMaxClass], ndim[kMaxClass], nstr[kMaxClass];
  int32_t pad[7];
};
static_assert(sizeof(TileRec) == 128, "tile record size");

__device__ __forceinline__ int32_t decomp(int32_t x, int n, const int32_t* dims, const int32_t* str) {
  int32_t off = 0;
  for(int j = n - 1; j >= 0; j--) {
    const int32_t d = dims[j], q = x / d;
    off += (x - q * d) * str[j];
    x = q;
  }
  return off;
}

// Offset of the k-th K element of a row: contiguous K (the inner labels are the
// trailing modes, last one stride 1) needs no index arithmetic.
__device__ __forceinline__ int32_t koff(const SplitBlock& b, int32_t k) {
  return b.kcontig ? k : decomp(k, b.nk, b.kdim, b.kstr);
}

constexpr int kPadRow = -0x7fffffff; // shift marker of a padding row (no digits)

// Row exponent e with |x| * 2^-e <= 127/128 for every x of the row, so that
// round(x * 2^(8S-1-e)) has a leading balanced digit within [-127, 127].
__device__ __forceinline__ int row_exponent(double mx) {
  int e = 0;
  if(mx > 0.0) {
    const double f = frexp(mx, &e); // mx = f * 2^e, f in [0.5, 1)
    if(f > 127.0 / 128.0) e += 1;
  }
  return e;
}


// round(x * 2^sh) + bias as a 64-bit word whose bytes are the balanced digits + 128.
// For S <= 6 (|X| < 2^47) one FMA against 1.5 * 2^52 leaves the integer, rounded to
// nearest even, in the low mantissa bits (2^52 + 2^51 + X); larger S convert directly.
template<int S>
__device__ __forceinline__ uint64_t digit_word(double x, double f, uint64_t bias) {
  if constexpr(S <= 6) {
    const uint64_t t = (uint64_t) __double_as_longlong(fma(x, f, 6755399441055744.0));
    return t + (bias - ((uint64_t) 1075 << 52) - ((uint64_t) 1 << 51));
  }
  else return (uint64_t) __double2ll_rn(x * f) + bias;
}

// Split in one pass over HBM: persistent CTAs, each taking 8-row groups ("chunks") in
// turn.  Phase 1, warp w streams row w
// (16-byte loads from the row's first 16-byte boundary, eight in flight per lane) for
// its max |x| and row exponent; phase 2 re-reads the 8 rows, now resident in L2, one
// 8-row x 16-k core matrix per warp and step: thread (row r, quad q) turns k =
// 4q..4q+3 into Y = round(x * 2^(8S-1-e)) + 0x80..80, whose plain base-256 bytes are
// the balanced digits + 128.  The bytes of 4 values are gathered per slice with PRMT,
// flipped back with one XOR and stored as one 4-byte word, so every warp store is a
// contiguous 128-byte core matrix.  Phase 2's re-reads and the digit stores are marked
// evict-first (streaming), so that the rows still waiting for their phase 2 keep L2.
// Slice layout per 32-byte K chunk of a tile: [K half (16 bytes)][digit][row][16 bytes],
// i.e. the S digits' core matrices of one K half follow each other, so that the digits
// j0..j1 of a B tile form one UMMA operand of (j1 - j0 + 1) x NT rows.  Residency (four CTAs per SM at 64 registers)
// bounds the rows held in L2 between the phases to 4 x 148 x 8 rows (87 MB at K =
// 2304, within the 126 MB L2).
//
// BF (the BF16x3 mode, S = 2): the row is scaled by 2^-e and each value x cut into two
// bf16 pieces, hi = bf16(x) and lo = bf16(x - hi) (round to nearest), in the same
// layout with 2-byte elements: a 16-byte core-matrix row holds 8 values, thread
// (row r, pair q) converts k = 2q, 2q+1 of an 8-value column.
template<int S, bool BF>
__global__ void __launch_bounds__(256) k_split_fused(const SplitBlock* __restrict__ blocks,
                                                     const int32_t* __restrict__ chunk_begin, int nblocks,
                                                     int nchunks,
                                                     const double* __restrict__ src, uint8_t* __restrict__ dst,
                                                     int32_t* __restrict__ exps, int32_t* __restrict__ blockmax) {
  __shared__ int     s_sh[8];
  __shared__ int32_t s_off[8];
  const int          warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t     bias = S >= 8 ? 0x8080808080808080ull : ((1ull << (8 * S)) - 1) / 255 * 128;
  // Block of chunk c: the last block whose first chunk is <= c (empty blocks skipped).
  // The next chunk of a CTA is usually a few blocks on, so each lane holds the first
  // chunk of one of the 32 blocks after the current one, loaded one chunk ahead (the
  // load is in flight while the current chunk is split); past them, a 32-way search
  // with one ballot per step keeps chunk_begin[lo] <= c < chunk_begin[hi], the lanes
  // probing lo + step .. lo + 32 step, of which those at or below c form a prefix.
  auto probe = [&](int from) {
    return from + 1 + lane < nblocks ? __ldg(chunk_begin + from + 1 + lane) : 0x7fffffff;
  };
  int lo = 0, next_first = probe(0); // chunk_begin[lo] <= c holds for every later c
  for(int c = blockIdx.x; c < nchunks; c += gridDim.x) {
    int hi;
    {
      const int cnt = __popc(__ballot_sync(0xffffffffu, next_first <= c));
      lo += cnt;
      hi = cnt < 32 ? lo + 1 : nblocks; // a failed probe at lo + 1 bounds the block
    }
    while(hi - lo > 1) {
      const int      step = (hi - lo + 31) >> 5, idx = lo + (lane + 1) * step;
      const unsigned le   = __ballot_sync(0xffffffffu, idx < hi && __ldg(chunk_begin + idx) <= c);
      const int      cnt  = __popc(le);
      hi                  = min(hi, lo + (cnt + 1) * step);
      lo += cnt * step;
    }
    const int2       ch = make_int2(lo, 8 * (c - __ldg(chunk_begin + lo)));
    const SplitBlock b  = blocks[ch.x];
    next_first          = probe(lo);
    {
      const int     row    = ch.y + warp;
      const bool    live   = row < b.rows;
      const int32_t rowoff = live ? decomp(row, b.nr, b.rdim, b.rstr) : 0;
      double        mx     = 0.0;
      if(live) {
        const double* s = src + b.src_off + rowoff;
        double        m[8];
#pragma unroll
        for(int x = 0; x < 8; x++) m[x] = 0.0;
        if(b.kcontig) {
          // 16-byte loads from the first 16-byte boundary of the row on
          const int      p0 = (reinterpret_cast<uintptr_t>(s) & 15) ? 1 : 0;
          const int      np = (b.K - p0) >> 1;
          const double2* s2 = reinterpret_cast<const double2*>(s + p0);
          int            k  = lane;
          for(; k + 224 < np; k += 256) {
            double2 t[8];
#pragma unroll
            for(int x = 0; x < 8; x++) t[x] = __ldg(s2 + k + 32 * x);
#pragma unroll
            for(int x = 0; x < 8; x++) m[x] = fmax(m[x], fmax(fabs(t[x].x), fabs(t[x].y)));
          }
          for(; k < np; k += 32) {
            const double2 t = __ldg(s2 + k);
            m[0]            = fmax(m[0], fmax(fabs(t.x), fabs(t.y)));
          }
          if(lane == 0 && p0) m[1] = fmax(m[1], fabs(__ldg(s)));
          if(lane == 1 && p0 + 2 * np < b.K) m[1] = fmax(m[1], fabs(__ldg(s + b.K - 1)));
        }
        else
          for(int k = lane; k < b.K; k += 32) m[0] = fmax(m[0], fabs(__ldg(s + koff(b, k))));
#pragma unroll
        for(int x = 0; x < 8; x++) mx = fmax(mx, m[x]);
      }
#pragma unroll
      for(int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      if(lane == 0) {
        const int e = row_exponent(mx);
        s_sh[warp]  = live ? (BF ? -e : 8 * S - 1 - e) : kPadRow;
        s_off[warp] = rowoff;
        exps[b.exp_off + row] = e;
        if(mx > 0.0) atomicMax(blockmax + b.id, e);
      }
    }
    __syncthreads();
    const int     r = lane >> 2, q = lane & 3; // row within the 8-row group, k quad
    const int     sh   = s_sh[r];
    const bool    live = sh != kPadRow;
    const double* s    = src + b.src_off + s_off[r];
    // 2^sh as two factors, so that no factor overflows for extreme row exponents
    const double f1  = ldexp(1.0, live ? sh / 2 : 0), f2 = ldexp(1.0, live ? sh - sh / 2 : 0);
    const int g8 = (ch.y % b.tile_rows) >> 3;
    if constexpr(BF) {
      const int nkc = b.K_pad * 2 / KC;
      uint8_t*  out = dst + b.dst_off + (int64_t) (ch.y / b.tile_rows) * nkc * S * b.tile_rows * KC + g8 * 128 +
                     r * 16 + q * 4;
      const bool vec = live && b.kcontig && !(reinterpret_cast<uintptr_t>(s) & 15);
      for(int k8 = warp; k8 < b.K_pad / 8; k8 += 8) {
        const int k0 = k8 * 8 + q * 2;
        double    v[2];
        if(vec && k0 + 1 < b.K) {
          const double2 v01 = __ldcs(reinterpret_cast<const double2*>(s + k0));
          v[0] = v01.x, v[1] = v01.y;
        }
        else
#pragma unroll
          for(int x = 0; x < 2; x++) v[x] = (live && k0 + x < b.K) ? __ldcs(s + koff(b, k0 + x)) : 0.0;
        uint32_t hi = 0, lo = 0;
#pragma unroll
        for(int x = 0; x < 2; x++) {
          const double         y = v[x] * f1 * f2;
          const __nv_bfloat16  h = __double2bfloat16(y);
          const __nv_bfloat16  t = __double2bfloat16(y - (double) __bfloat162float(h));
          hi |= (uint32_t) __bfloat16_as_ushort(h) << (16 * x);
          lo |= (uint32_t) __bfloat16_as_ushort(t) << (16 * x);
        }
        uint8_t* o = out + (int64_t) (k8 >> 1) * S * b.tile_rows * KC + (k8 & 1) * S * b.tile_rows * 16;
        __stcs(reinterpret_cast<unsigned int*>(o), hi);
        __stcs(reinterpret_cast<unsigned int*>(o + b.tile_rows * 16), lo);
      }
    }
    else {
      const int    nkc = b.K_pad / KC;
      uint8_t* out = dst + b.dst_off + (int64_t) (ch.y / b.tile_rows) * nkc * S * b.tile_rows * KC + g8 * 128 + r * 16 +
                     q * 4;
      const bool vec = live && b.kcontig && !(reinterpret_cast<uintptr_t>(s) & 15);
      // loads of one 16-value column (this thread's row and quad) and the conversion
      // of it into S 4-byte digit words; two columns per iteration keep the second
      // column's loads in flight while the first converts
      auto load4 = [&](int k16, double (&v)[4]) {
        const int k0 = k16 * 16 + q * 4;
        if(vec && k0 + 3 < b.K) {
          const double2 v01 = __ldcs(reinterpret_cast<const double2*>(s + k0));
          const double2 v23 = __ldcs(reinterpret_cast<const double2*>(s + k0 + 2));
          v[0] = v01.x, v[1] = v01.y, v[2] = v23.x, v[3] = v23.y;
        }
        else
#pragma unroll
          for(int x = 0; x < 4; x++) {
            const int k = k0 + x;
            v[x]        = (live && k < b.K) ? __ldcs(s + koff(b, k)) : 0.0;
          }
      };
      auto emit = [&](int k16, const double (&v)[4]) {
        uint32_t lo[4], hi[4];
#pragma unroll
        for(int x = 0; x < 4; x++) {
          const uint64_t Y = digit_word<S>(v[x] * f2, f1, bias);
          lo[x]            = (uint32_t) Y;
          hi[x]            = (uint32_t) (Y >> 32);
        }
        uint8_t* o = out + (int64_t) (k16 >> 1) * S * b.tile_rows * KC + (k16 & 1) * S * b.tile_rows * 16;
#pragma unroll
        for(int i = 0; i < S; i++) {
          const int p = S - 1 - i; // byte of Y holding digit i
          uint32_t  w;
          if(p < 4) {
            const uint32_t t0 = __byte_perm(lo[0], lo[1], p | ((p + 4) << 4));
            const uint32_t t1 = __byte_perm(lo[2], lo[3], p | ((p + 4) << 4));
            w                 = __byte_perm(t0, t1, 0x5410);
          }
          else {
            const uint32_t t0 = __byte_perm(hi[0], hi[1], (p - 4) | (p << 4));
            const uint32_t t1 = __byte_perm(hi[2], hi[3], (p - 4) | (p << 4));
            w                 = __byte_perm(t0, t1, 0x5410);
          }
          __stcs(reinterpret_cast<unsigned int*>(o + (int64_t) i * b.tile_rows * 16), w ^ 0x80808080u);
        }
      };
      const int n16 = b.K_pad / 16;
      for(int k16 = warp; k16 < n16; k16 += 16) {
        double v0[4], v1[4];
        load4(k16, v0);
        const bool two = k16 + 8 < n16;
        if(two) load4(k16 + 8, v1);
        emit(k16, v0);
        if(two) emit(k16 + 8, v1);
      }
    }
    __syncthreads(); // s_sh / s_off are rewritten for the next chunk
  }
}

// Staged split for operand blocks whose rows lie one after another in memory (K
// contiguous and row r at element offset r * K: e.g. v(a,b,c,d) split as rows (a,b) by
// K = (c,d)).  The unit of work is a pair of rows, one contiguous range of 2K doubles,
// brought into shared memory by one bulk copy; every element is read from HBM once, and
// both the row maxima and the digit conversion read shared memory.
//   Producer (warp 0): resolves 32 units at a time, one per lane (block by binary
// search over the per-block chunk prefix, then the unit's copy range and the fields the
// consumers need), and issues their copies in order into the stage of the group that
// takes each unit.  A CTA owns whole 8-row chunks: the four units of a chunk fill the
// same 128-byte lines of every digit plane, and lines completed by one SM within a
// short time leave L2 whole (units spread over SMs measured 1.4x slower at the size
// of the O=40/V=360 ladder's v, while as fast on a quarter of it).  The unit records
// travel in shared memory beside the stages, so a consumer reads no block record from
// global memory.
//   Consumers: independent groups of kSplitGroup warps, each group with two stages of
// its own, so a group's only synchronisation is a named barrier of its own warps.
// Warp h of a group takes the h-th K range of the row maxima and every kSplitGroup-th
// group of four 16-k chunks of the digits.  Lane (row, chunk c, quad q) reads its four
// values in an order rotated by (q + c) mod 4, so that the 16 lanes of a row hit 16
// distinct bank pairs, and the final byte permute puts the digits back in k order;
// each warp store covers the two rows of 32-byte sectors.
//   The copy covers the 16-byte aligned interior [floor16(start), floor16(end)) of the
// pair; a last element past floor16(end) is loaded with a plain load.  Units made of
// padding rows only write their exponents.  Waits are bounded: a timeout records
// `code` in *err and the warps of a group agree (bar.red) to leave together.
struct UnitMeta {
  int64_t tail_src; // element index of the unit's last element (the tail load)
  int64_t dst_off;  // byte offset of the block's digits
  int32_t exp_base; // exponent index of the unit's first row
  int32_t id, K, K_pad, tile_rows, row0, nlive, delta, tail;
  int32_t pad[3];
};
static_assert(sizeof(UnitMeta) == 64, "unit record size");

constexpr int     kSplitGroup     = 4;            // consumer warps per group
constexpr int     kSplitMaxGroups = 4;            // groups per CTA, at most
constexpr int64_t kStagedSmem     = 227 * 1024;   // dynamic shared memory of one CTA, at most
constexpr int64_t kStagedHead     = 2048;         // barriers, unit records, partial maxima
// bytes of one stage of 2 rows of K doubles (+16 for the aligned start), 128-byte multiple
__host__ __device__ constexpr int64_t staged_stage_bytes(int64_t K) {
  return (2 * K * 8 + 16 + 127) / 128 * 128;
}

// TR: rows per operand tile (128 for A; 0 = read from the unit record).
template<int S, int TR>
__global__ void __launch_bounds__(32 * (1 + kSplitMaxGroups * kSplitGroup), 1)
  k_split_staged(const SplitBlock* __restrict__ blocks, const int32_t* __restrict__ chunk_begin, int nblocks,
                 int nchunks, int ngroups, uint32_t stage_bytes, const double* __restrict__ src,
                 uint8_t* __restrict__ dst, int32_t* __restrict__ exps, int32_t* __restrict__ blockmax, int* err) {
  constexpr int G = kSplitGroup;
  extern __shared__ __align__(128) uint8_t sm[];
  uint64_t*     full  = reinterpret_cast<uint64_t*>(sm);           // [2 per group]
  uint64_t*     empty = full + 2 * kSplitMaxGroups;                // [2 per group]
  UnitMeta*     meta  = reinterpret_cast<UnitMeta*>(sm + 256);     // [2 per group]
  double*       part  = reinterpret_cast<double*>(sm + 1280);      // [group][parity][warp][row]
  uint8_t*      ring  = sm + kStagedHead;
  static_assert(4 * kSplitMaxGroups * 8 <= 256 && 256 + 2 * kSplitMaxGroups * 64 <= 1280, "stage records");
  static_assert(1280 + 2 * kSplitMaxGroups * G * 2 * 8 <= kStagedHead, "partial maxima");
  const int     warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int     nunits = nchunks * 4; // two rows per unit, four units per 8-row chunk
  // units of this CTA: the four of each of its chunks
  const int     myunits = ((nchunks - (int) blockIdx.x + (int) gridDim.x - 1) / (int) gridDim.x) * 4;
  if(threadIdx.x == 0) {
    for(int x = 0; x < 2 * ngroups; x++) {
      mbar_init(&full[x], 1);
      mbar_init(&empty[x], G); // one arrival per warp of the group
    }
    fence_mbarrier_init();
  }
  __syncthreads();
  if(warp == 0) {
    // ---------------- producer: 32 unit records at a time, copies in unit order -------
    // The CTA's j-th unit is unit j mod 4 of 8-row chunk blockIdx.x + (j / 4) * gridDim.x
    // (the four units of a chunk, whose digits share every 128-byte line, are written
    // by one SM close together in time); it goes to group j mod ngroups, that group's
    // stage (j / ngroups) mod 2.
    for(int jb = 0; jb < myunits; jb += 32) {
      const int jl = jb + lane;
      const int u  = jl < myunits ? ((int) blockIdx.x + (jl >> 2) * (int) gridDim.x) * 4 + (jl & 3) : nunits;
      UnitMeta  mine{};
      uintptr_t a16   = 0;
      uint32_t  bytes = 0;
      if(u < nunits) {
        const int c = u >> 2;
        int       lo = 0, hi = nblocks - 1; // last block whose first chunk is <= c
        while(lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if(__ldg(chunk_begin + mid) <= c) lo = mid;
          else hi = mid - 1;
        }
        const SplitBlock& b    = blocks[lo];
        const int         row0 = 8 * (c - __ldg(chunk_begin + lo)) + (u & 3) * 2;
        const int         K    = b.K;
        const int         nl   = max(0, min(2, b.rows - row0));
        mine.dst_off   = b.dst_off;
        mine.exp_base  = b.exp_off + row0;
        mine.id        = b.id;
        mine.K         = K;
        mine.K_pad     = b.K_pad;
        mine.tile_rows = b.tile_rows;
        mine.row0      = row0;
        mine.nlive     = nl;
        mine.tail_src  = b.src_off + (int64_t) (row0 + nl) * K - 1;
        if(nl > 0) {
          const uintptr_t start = reinterpret_cast<uintptr_t>(src + b.src_off + (int64_t) row0 * K);
          const uintptr_t end   = start + (uintptr_t) nl * K * 8;
          a16                   = start & ~uintptr_t(15);
          bytes                 = (uint32_t) ((end & ~uintptr_t(15)) - a16);
          mine.delta            = (int32_t) (start - a16);
          mine.tail             = (end & 15) ? 1 : 0;
        }
      }
      for(int t = 0; t < 32; t++) {
        if(jb + t >= myunits) break;
        const int      j     = jb + t;
        const int      x     = 2 * (j % ngroups) + ((j / ngroups) & 1);
        const uint32_t round = (uint32_t) (j / (2 * ngroups));
        if(!mbar_wait(&empty[x], (round & 1) ^ 1, err, 21)) return; // (every lane polls; all agree)
        if(lane == t) {
          meta[x] = mine;
          mbar_arrive_expect_tx(&full[x], bytes);
          if(bytes > 0)
            bulk_g2s(ring + (size_t) x * stage_bytes, reinterpret_cast<const void*>(a16), bytes, &full[x]);
        }
        __syncwarp();
      }
    }
    return;
  }
  // ---------------- consumers: groups of G warps ----------------
  const int cw = warp - 1, grp = cw / G, h = cw % G;
  if(grp >= ngroups) return;
  const int      barid = 1 + grp; // named barrier of the group (0 is __syncthreads)
  const uint64_t bias  = S >= 8 ? 0x8080808080808080ull : ((1ull << (8 * S)) - 1) / 255 * 128;
  const int      rr = lane >> 4, c = (lane >> 2) & 3, q = lane & 3; // row of the pair, chunk, quad
  const int      rot = (q + c) & 3;
  uint32_t       sel2 = 0; // byte permute taking the rotated values back to k order
#pragma unroll
  for(int pos = 0; pos < 4; pos++) {
    const int t = (pos - rot) & 3;
    sel2 |= (uint32_t) (t < 2 ? t : t + 2) << (4 * pos);
  }
  for(int j = grp; j < myunits; j += ngroups) {
    const int      par   = (j / ngroups) & 1, x = 2 * grp + par;
    const uint32_t round = (uint32_t) (j / (2 * ngroups));
    {
      const bool got = mbar_wait(&full[x], round & 1, err, 22);
      uint32_t   anyfail;
      asm volatile("{\n\t.reg .pred p, q;\n\tsetp.eq.u32 p, %1, 0;\n\t"
                   "bar.red.or.pred q, %2, %3, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
                   : "=r"(anyfail)
                   : "r"((uint32_t) got), "r"(barid), "n"(32 * G)
                   : "memory");
      if(anyfail) return;
    }
    const UnitMeta m       = meta[x];
    const int      K       = m.K;
    const int      tr      = TR > 0 ? TR : m.tile_rows;
    double*        rowbase = reinterpret_cast<double*>(ring + (size_t) x * stage_bytes + m.delta);
    if(m.tail) { // the last element, past the copy's 16-byte aligned end
      if(h == 0 && lane == 0) {
        rowbase[(int64_t) m.nlive * K - 1] = __ldg(src + m.tail_src);
        // ordered before the bulk copy that later refills this stage
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      }
      asm volatile("bar.sync %0, %1;\n" ::"r"(barid), "n"(32 * G) : "memory");
    }
    // row maxima: 16 lanes per row over this warp's K range, then over the group
    const double* xr   = rowbase + (int64_t) rr * K;
    const bool    live = rr < m.nlive;
    double        mx   = 0.0;
    if(live) {
      const int span = (K + G - 1) / G, kb = h * span, ke = min(K, kb + span);
      double    m0 = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0;
      int       k = kb + (lane & 15);
      for(; k + 48 < ke; k += 64) {
        m0 = fmax(m0, fabs(xr[k]));
        m1 = fmax(m1, fabs(xr[k + 16]));
        m2 = fmax(m2, fabs(xr[k + 32]));
        m3 = fmax(m3, fabs(xr[k + 48]));
      }
      for(; k < ke; k += 16) m0 = fmax(m0, fabs(xr[k]));
      mx = fmax(fmax(m0, m1), fmax(m2, m3));
    }
#pragma unroll
    for(int o = 8; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    // partials alternate between two buffers by unit parity: a warp writes this buffer
    // again only after the group's next barrier, which every reader of it has passed
    double* pp = part + (grp * 2 + par) * G * 2;
    if((lane & 15) == 0) pp[h * 2 + rr] = mx;
    asm volatile("bar.sync %0, %1;\n" ::"r"(barid), "n"(32 * G) : "memory");
    mx = 0.0;
#pragma unroll
    for(int w = 0; w < G; w++) mx = fmax(mx, pp[w * 2 + rr]);
    const int e = row_exponent(mx);
    if(h == 0 && (lane & 15) == 0) {
      exps[m.exp_base + rr] = e;
      if(mx > 0.0) atomicMax(blockmax + m.id, e);
    }
    if(m.nlive > 0) {
      // digits: 2^sh in one factor where it is a normal double, else as two (tiny rows)
      const int     sh   = live ? 8 * S - 1 - e : 0;
      const bool    wide = sh > 1000 || sh < -1000;
      const double  f1 = ldexp(1.0, wide ? sh / 2 : sh), f2 = ldexp(1.0, wide ? sh - sh / 2 : 0);
      const int     row   = m.row0 + rr;
      const int     nkc   = m.K_pad / KC;
      const int64_t dstep = (int64_t) S * tr * 16; // one K half of a 32-byte K chunk
      uint8_t*      o = dst + m.dst_off + (int64_t) (row / tr) * nkc * S * tr * KC + ((row % tr) >> 3) * 128 +
                   (row & 7) * 16 + q * 4 + ((c >> 1) * 2 + (c & 1) + (int64_t) h * 4) * dstep;
      const int     n16     = m.K_pad / 16;
      const bool    anywide = __any_sync(0xffffffffu, wide && live);
      for(int k16 = 4 * h + c; k16 < n16; k16 += 4 * G, o += 4 * G * dstep) {
        const int k0 = k16 * 16 + q * 4;
        double    v[4];
#pragma unroll
        for(int t = 0; t < 4; t++) {
          const int kk = k0 + ((t + rot) & 3);
          v[t]         = (live && kk < K) ? xr[kk] : 0.0;
        }
        if(anywide)
#pragma unroll
          for(int t = 0; t < 4; t++) v[t] *= f2;
        uint32_t lo[4], hi[4];
#pragma unroll
        for(int t = 0; t < 4; t++) {
          const uint64_t Y = digit_word<S>(v[t], f1, bias);
          lo[t]            = (uint32_t) Y;
          hi[t]            = (uint32_t) (Y >> 32);
        }
#pragma unroll
        for(int i = 0; i < S; i++) {
          const int p = S - 1 - i; // byte of Y holding digit i
          uint32_t  t0, t1;
          if(p < 4) {
            t0 = __byte_perm(lo[0], lo[1], p | ((p + 4) << 4));
            t1 = __byte_perm(lo[2], lo[3], p | ((p + 4) << 4));
          }
          else {
            t0 = __byte_perm(hi[0], hi[1], (p - 4) | (p << 4));
            t1 = __byte_perm(hi[2], hi[3], (p - 4) | (p << 4));
          }
          __stcs(reinterpret_cast<unsigned int*>(o + (int64_t) i * tr * 16), __byte_perm(t0, t1, sel2) ^ 0x80808080u);
        }
      }
    }
    __syncwarp();
    if(lane == 0) mbar_arrive(&empty[x]); // this warp is done with the stage
  }
}

// Slice count per task: a task whose largest possible product (2^(maxexp A + maxexp
// B) * K) is 2^(8m) below the largest of its output group needs m fewer digits for
// the same absolute truncation error; numerically zero blocks keep one digit.
// One warp per output group, lanes over its tasks.
__global__ void k_task_slices(const I8TaskMeta* __restrict__ meta, const DevGroup* __restrict__ groups,
                              int ngroups, const int32_t* __restrict__ amax, const int32_t* __restrict__ bmax,
                              int smax, uint8_t* __restrict__ tslices) {
  constexpr int kNone = -1000000; // blockmax slots start at 0x80808080 (no nonzero row)
  const int     lane  = threadIdx.x & 31;
  for(int gi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; gi < ngroups; gi += (gridDim.x * blockDim.x) >> 5) {
    const DevGroup g  = groups[gi];
    int            eg = kNone;
    for(int t = g.task_begin + lane; t < g.task_end; t += 32) {
      const int ea = amax[meta[t].a_block], eb = bmax[meta[t].b_block];
      if(ea > kNone && eb > kNone) eg = max(eg, ea + eb + meta[t].log2k);
    }
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) eg = max(eg, __shfl_xor_sync(0xffffffffu, eg, o));
    for(int t = g.task_begin + lane; t < g.task_end; t += 32) {
      const int ea = amax[meta[t].a_block], eb = bmax[meta[t].b_block];
      int       s  = 1;
      if(ea > kNone && eb > kNone) s = max(1, smax - (eg - (ea + eb + meta[t].log2k)) / 8);
      tslices[t] = (uint8_t) s;
    }
  }
}

struct I8Params {
  const uint8_t*  a_slices; // digit slices of the A blocks (task a_off is relative to it)
  const uint8_t*  b_slices;
  const int32_t*  a_exps;   // row exponents (task a_exp / b_exp relative to these)
  const int32_t*  b_exps;
  const I8Task*   tasks;
  const DevGroup* groups;
  const I8Item*   items;
  int             nitems;
  double*         C;
  double          alpha;
  LabelClasses    lc;
  int*            err;
  const uint8_t*  tslices; // digit count of each task (1..S)
  int*            ctr;     // next output tile to hand out (zero at launch)
  int             xpose;   // C is contiguous along the tile's columns: transposed reductions
  int             store;   // C = alpha * result (an assignment whose output blocks this
                           // launch covers completely) instead of C += alpha * result
  int             energy = 0; // set for the EN instantiations: sum (C + alpha * result)^2 / D into en.part
  EnergyArgs      en;
};

template<int S, int NT>
__host__ __device__ constexpr uint32_t stage_bytes() {
  return (uint32_t) S * (MT + NT) * KC;
}

constexpr int kTail  = 4608; // barriers, column scales, C offsets and tile records behind the stages
constexpr int kTailD = 2560; // offset in the tail of the columns' denominator parts (2 x NT doubles)
constexpr int kTailT = 3840; // offset in the tail of the queue slots' tile records
constexpr int kQueue = 4;    // output tiles in flight between producer, MMA issuer and epilogue

// Pipeline depth: as many stages as fit beside the tail, at most 6.
template<int S, int NT>
__host__ __device__ constexpr int stages() {
  return (int) ((kMaxSmem - kTail) / stage_bytes<S, NT>()) < 6 ? (int) ((kMaxSmem - kTail) / stage_bytes<S, NT>()) : 6;
}

// Epilogue transpose buffer behind the tail, where it fits: per epilogue warp XC (8 or
// 4) columns x 32 rows of doubles, rows kXStride apart (34: the transposed reads of a half
// warp, 8 columns x 2 rows, fall on 16 distinct bank pairs), 64 columns in all: eight
// warps of 8 columns, or sixteen of 4.
constexpr int kXStride = 34;
constexpr int kXBytes = 64 * kXStride * 8;
template<int S, int NT>
__host__ __device__ constexpr bool xpose_fits() {
  return (size_t) stages<S, NT>() * stage_bytes<S, NT>() + kTail + kXBytes <= kMaxSmem;
}

template<int S, int NT>
constexpr size_t smem_bytes() {
  return (size_t) stages<S, NT>() * stage_bytes<S, NT>() + kTail + (xpose_fits<S, NT>() ? kXBytes : 0);
}

// BF: the BF16x3 mode (S = 2 bf16 pieces, kind::f16 MMAs with FP32 accumulators; both
// diagonals carry the same power of two, 2^(e_row + e_col)).
// EN: the energy epilogue (p.energy) instead of the C update, in instantiations of its
// own so that the plain kernels' code is unchanged.
// EW: epilogue warps, 8 or 16 (four per TMEM lane quarter, each a quarter of the tile's
// columns: for contractions whose tiles have little K, where the epilogue bounds the
// kernel; the threads then get at most 96 registers each).
template<int S, int NT, bool BF, bool EN = false, int EW = 8>
__global__ void __launch_bounds__(64 + 32 * EW, 1) k_contract_i8(const I8Params p) {
  static_assert(S * NT <= 512, "TMEM holds 512 columns");
  static_assert(EW == 8 || (EW == 16 && !EN && !BF), "sixteen epilogue warps: the plain INT8 C update only");
  constexpr int NE = 32 * EW; // epilogue threads
  extern __shared__ __align__(1024) uint8_t smem[];
  constexpr uint32_t A_BYTES = S * MT * KC, B_BYTES = S * NT * KC, STAGE = A_BYTES + B_BYTES;
  constexpr int      kStack  = 256 / NT; // B digits per MMA (UMMA N <= 256)
  static_assert(kStack >= 3, "a drain group's three B digits fit one MMA");
  constexpr int      STAGES  = stages<S, NT>();
  static_assert(STAGES >= 2, "two pipeline stages at least");
  uint64_t*          full   = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE);
  uint64_t*          empty  = full + STAGES;
  uint64_t*          tfull  = empty + STAGES;
  uint64_t*          tempty = tfull + 1;                                    // one per diagonal
  uint64_t*          qfull  = tempty + 8;                                    // tile queue
  uint64_t*          qempty = qfull + kQueue;
  double*            sc     = reinterpret_cast<double*>(qempty + kQueue);    // column scales, 2 x NT
  int32_t*           noff   = reinterpret_cast<int32_t*>(sc + 2 * NT);       // C column offsets, 2 x NT
  int32_t*           qitem  = noff + 2 * NT;
  uint32_t*          tslot  = reinterpret_cast<uint32_t*>(qitem + kQueue);
  double*            dcol   = reinterpret_cast<double*>(smem + STAGES * STAGE + kTailD); // 2 x NT
  TileRec*           trec   = reinterpret_cast<TileRec*>(smem + STAGES * STAGE + kTailT);  // kQueue
  static_assert(sizeof(uint64_t) * (2 * 6 + 1 + 8 + 2 * kQueue) + (sizeof(double) + sizeof(int32_t)) * 2 * NT +
                    4 * kQueue + 4 <=
                  kTailD,
                "shared-memory tail");
  static_assert(kTailD + sizeof(double) * 2 * NT <= kTailT, "shared-memory tail (denominators)");
  static_assert(kTailT + sizeof(TileRec) * kQueue <= kTail, "shared-memory tail (tile records)");
  const int          warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if(threadIdx.x == 0) {
    for(int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(tfull, 1);
    for(int d = 0; d < S; d++) mbar_init(&tempty[d], NE);
    for(int i = 0; i < kQueue; i++) {
      mbar_init(&qfull[i], 1);
      mbar_init(&qempty[i], 1 + NE); // the MMA issuer and every epilogue thread
    }
    fence_mbarrier_init();
  }
  if(warp == 1) tmem_alloc(tslot, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  if(warp == 0) {
    // ---------------- producer: one bulk copy of all S digit slices per operand ----
    if(elect_one()) {
      int      stage = 0;
      uint32_t phase = 0;
      int       qslot = 0;
      uint32_t  qph   = 0;
      while(true) { // tiles are handed out longest first, to whichever CTA is free
        if(!mbar_wait(&qempty[qslot], qph ^ 1, p.err, 5)) goto done_producer;
        const int it = atomicAdd(p.ctr, 1);
        qitem[qslot] = it < p.nitems ? it : -1;
        I8Item   item{};
        DevGroup g{};
        if(it < p.nitems) {
          item       = p.items[it];
          g          = p.groups[item.group];
          TileRec& r = trec[qslot];
          r.c_off      = g.c_off;
          r.group      = item.group;
          r.mt         = item.mt;
          r.nt         = item.nt;
          r.task_begin = g.task_begin;
          r.task_end   = g.task_end;
          int32_t cstr[kMaxModes]; // C block strides (a block holds fewer than 2^31 elements)
          int32_t sz = 1;
          for(int i = p.lc.nc - 1; i >= 0; i--) {
            cstr[i] = sz;
            sz *= g.cdims[i];
          }
          int32_t M = 1, N = 1;
          for(int j = 0; j < p.lc.nm; j++) {
            r.mdim[j] = g.cdims[p.lc.m_c[j]];
            r.mstr[j] = cstr[p.lc.m_c[j]];
            M *= r.mdim[j];
          }
          for(int j = 0; j < p.lc.nn; j++) {
            r.ndim[j] = g.cdims[p.lc.n_c[j]];
            r.nstr[j] = cstr[p.lc.n_c[j]];
            N *= r.ndim[j];
          }
          r.M = M;
          r.N = N;
          if(g.task_begin < g.task_end) { // the first task's row exponents and column scales, to L1
            const I8Task   t0 = p.tasks[g.task_begin];
            const int32_t* ea = p.a_exps + t0.a_exp + item.mt * MT;
            const int32_t* eb = p.b_exps + t0.b_exp + item.nt * NT;
#pragma unroll
            for(int o = 0; o < MT; o += 32) asm volatile("prefetch.global.L1 [%0];\n" ::"l"(ea + o));
            asm volatile("prefetch.global.L1 [%0];\n" ::"l"(ea + MT - 1));
#pragma unroll
            for(int o = 0; o < NT; o += 32) asm volatile("prefetch.global.L1 [%0];\n" ::"l"(eb + o));
            asm volatile("prefetch.global.L1 [%0];\n" ::"l"(eb + NT - 1));
          }
        }
        mbar_arrive(&qfull[qslot]); // (release: the record is visible to the slot's waiters)
        if(++qslot == kQueue) {
          qslot = 0;
          qph ^= 1;
        }
        if(it >= p.nitems) break;
        for(int t = g.task_begin; t < g.task_end; t++) {
          const I8Task   tk = p.tasks[t];
          const uint8_t* ga = p.a_slices + tk.a_off + (int64_t) item.mt * tk.nkc * A_BYTES;
          const uint8_t* gb = p.b_slices + tk.b_off + (int64_t) item.nt * tk.nkc * B_BYTES;
          const uint32_t st = p.tslices[t]; // only the task's leading digits travel
          const uint32_t ab = st * MT * 16, bb = st * NT * 16; // per K half
          for(int kc = 0; kc < tk.nkc; kc++) {
            if(!mbar_wait(&empty[stage], phase ^ 1, p.err, 1)) goto done_producer;
            mbar_arrive_expect_tx(&full[stage], 2 * (ab + bb));
            uint8_t*       sa = smem + stage * STAGE;
            const uint8_t* ka = ga + (int64_t) kc * A_BYTES;
            const uint8_t* kb = gb + (int64_t) kc * B_BYTES;
            if(st == S) { // both K halves in one copy per operand
              bulk_g2s(sa, ka, A_BYTES, &full[stage]);
              bulk_g2s(sa + A_BYTES, kb, B_BYTES, &full[stage]);
            }
            else
              for(int h = 0; h < 2; h++) {
                bulk_g2s(sa + h * (A_BYTES / 2), ka + h * (A_BYTES / 2), ab, &full[stage]);
                bulk_g2s(sa + A_BYTES + h * (B_BYTES / 2), kb + h * (B_BYTES / 2), bb, &full[stage]);
              }
            if(++stage == STAGES) {
              stage = 0;
              phase ^= 1;
            }
          }
        }
      }
    done_producer:;
    }
  }
  else if(warp == 1) {
    // ------- MMA issuer: S(S+1)/2 digit products per K step in stacked-B MMAs --------
    if(elect_one()) {
      int      stage = 0;
      uint32_t phase = 0, tphase = 0;
      int       qslot = 0;
      uint32_t  qph   = 0;
      while(true) {
        if(!mbar_wait(&qfull[qslot], qph, p.err, 6)) goto done_mma;
        const int it = qitem[qslot];
        int       tb = 0, te = 0;
        if(it >= 0) {
          tb = trec[qslot].task_begin;
          te = trec[qslot].task_end;
        }
        mbar_arrive(&qempty[qslot]);
        if(++qslot == kQueue) {
          qslot = 0;
          qph ^= 1;
        }
        if(it < 0) break;
        for(int t = tb; t < te; t++) {
          const int nkc = p.tasks[t].nkc;
          const int st  = p.tslices[t];
          for(int kc = 0; kc < nkc; kc++) {
            if(!mbar_wait(&full[stage], phase, p.err, 3)) goto done_mma;
            tc_fence_after();
            const uint32_t a0 = smem_u32(smem + stage * STAGE), b0 = a0 + A_BYTES;
            // A digit i times the stacked B digits j0 .. j0 + nd - 1 in one MMA of N =
            // nd * NT: it adds into the adjacent diagonals i + j0 .. i + j0 + nd - 1
            if(kc == 0) {
              // First K step of a task: the previous task's diagonals must have been read
              // out.  The products go by the epilogue's drain groups of three diagonals
              // (the same S(S+1)/2 products in as many MMAs), so those into diagonals 0-2
              // start as soon as the epilogue has read the first group; in each group the
              // A digit 0 product comes first and overwrites, the others accumulate.
              int waited = 0;
#pragma unroll
              for(int g0 = 0; g0 < S; g0 += 3) {
                const int gl = S - g0 < 3 ? S - g0 : 3;
                for(; waited < g0 + gl; waited++) {
                  if(!mbar_wait(&tempty[waited], tphase ^ 1, p.err, 2)) goto done_mma;
                  tc_fence_after();
                }
#pragma unroll
                for(int i = 0; i < S; i++) {
                  if(i >= st || i > g0 + gl - 1) break;
                  const int jlo = g0 - i > 0 ? g0 - i : 0;
                  const int jhi = min(g0 + gl - 1 - i, st - 1 - i);
                  if(jlo > jhi) continue;
                  const int      nd = jhi - jlo + 1; // <= 3 <= kStack
                  const uint64_t ad = umma_desc_kmajor(a0 + i * MT * 16, S * MT * 16, 128);
                  const uint64_t bd = umma_desc_kmajor(b0 + jlo * NT * 16, S * NT * 16, 128);
                  if constexpr(BF) mma_f16(tmem + (i + jlo) * NT, ad, bd, idesc_bf16(MT, nd * NT), i > 0);
                  else mma_i8(tmem + (i + jlo) * NT, ad, bd, idesc_i8(MT, nd * NT, true, true), i > 0);
                }
              }
            }
            else {
#pragma unroll
              for(int i = 0; i < S; i++) {
                if(i >= st) break;
                const uint64_t ad = umma_desc_kmajor(a0 + i * MT * 16, S * MT * 16, 128);
#pragma unroll
                for(int j0 = 0; j0 < S; j0 += kStack) {
                  if(j0 >= st - i) break;
                  const int      nd = min(kStack, st - i - j0);
                  const uint64_t bd = umma_desc_kmajor(b0 + j0 * NT * 16, S * NT * 16, 128);
                  if constexpr(BF) mma_f16(tmem + (i + j0) * NT, ad, bd, idesc_bf16(MT, nd * NT), true);
                  else mma_i8(tmem + (i + j0) * NT, ad, bd, idesc_i8(MT, nd * NT, true, true), true);
                }
              }
            }
            umma_commit(&empty[stage]); // stage free once these MMAs have read it
            if(++stage == STAGES) {
              stage = 0;
              phase ^= 1;
            }
          }
          umma_commit(tfull); // the task's diagonals are complete
          tphase ^= 1;
        }
      }
    done_mma:;
    }
  }
  else {
    // ---------------- epilogue: FP64 recombination of the diagonals ----------------
    // EW warps: warp w reads TMEM lanes 32 * (w % 4) (its rows) and one of EW / 4 equal
    // column ranges of the tile, so EW / 4 warps share every lane quarter.
    constexpr int NH = NT / (EW / 4);
    // transpose width: 8 columns where the buffer holds 8 per warp, else 4
    constexpr int XC = (NH % 8 == 0 && EW * 8 <= 64) ? 8 : 4;
    static_assert(EW * XC <= 64 && NH % XC == 0, "transpose buffer");
    const int     q = warp & 3, row = q * 32 + lane, col0 = ((warp - 2) >> 2) * NH;
    const int     et = threadIdx.x - 64; // column whose scale this thread loads
    uint32_t      tphase = 0, tcount = 0, icount = 0;
    double        racc[NH];
    int           qslot = 0;
    uint32_t      qph   = 0;
    for(;; icount++) {
      int it, rslot;
      {
        // the epilogue threads agree on a timeout, so none is left in a barrier
        const bool got = mbar_wait(&qfull[qslot], qph, p.err, 7);
        uint32_t   anyfail;
        asm volatile("{\n\t.reg .pred p, q;\n\tsetp.eq.u32 p, %1, 0;\n\t"
                     "bar.red.or.pred q, 1, %2, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
                     : "=r"(anyfail)
                     : "r"((uint32_t) got), "n"(NE)
                     : "memory");
        if(anyfail) break;
        it    = qitem[qslot];
        rslot = qslot;
        if(++qslot == kQueue) {
          qslot = 0;
          qph ^= 1;
        }
      }
      if(it < 0) {
        mbar_arrive(&qempty[rslot]);
        break;
      }
      // the tile's record: read in shared memory while the C addressing is set up, then
      // the slot goes back to the producer
      const TileRec& rec = trec[rslot];
      const int      imt = rec.mt, int_ = rec.nt, igroup = rec.group, tb = rec.task_begin, te = rec.task_end;
#pragma unroll
      for(int x = 0; x < NH; x++) racc[x] = 0.0;
      bool ok = true;
      // C addressing of the tile (transpose_output fused: C's own label order),
      // computed while the tile's first task runs: the thread's row offset, and the
      // tile's column offsets in shared memory (alternating buffers by tile; the first
      // task's barrier below publishes them, the readers two tiles back are done)
      int64_t  rowoff = -1;
      double   drow   = 0.0; // energy epilogue: the row's part of the denominators
      int32_t* nof    = noff + (icount & 1) * NT;
      double*  dco    = dcol + (icount & 1) * NT;
      {
        const int      m  = imt * MT + row;
        const int32_t* es = p.en.estart + (int64_t) igroup * p.lc.nc;
        if(m < rec.M) {
          rowoff = rec.c_off + decomp(m, p.lc.nm, rec.mdim, rec.mstr);
          if constexpr(EN) drow = energy_part(m, p.lc.nm, rec.mdim, p.lc.m_c, p.en, es);
        }
        if(et < NT) {
          const int n = int_ * NT + et;
          nof[et]     = n < rec.N ? decomp(n, p.lc.nn, rec.ndim, rec.nstr) : -1;
          if constexpr(EN) dco[et] = n < rec.N ? energy_part(n, p.lc.nn, rec.ndim, p.lc.n_c, p.en, es) : 1.0;
        }
      }
      mbar_arrive(&qempty[rslot]);
      if constexpr(EN) {
        // the tile's C values go to L2 while its MMAs run (the energy epilogue reads them
        // once they are done): the epilogue warps publish the column offsets first
        asm volatile("bar.sync 1, %0;\n" ::"n"(NE) : "memory");
        if(rowoff >= 0) {
          const double* crow = p.C + rowoff;
#pragma unroll
          for(int x = 0; x < NH; x += (p.xpose ? XC : 1)) { // xpose: a row's columns are contiguous
            const int o = nof[col0 + x];
            if(o >= 0) asm volatile("prefetch.global.L2 [%0];\n" ::"l"(crow + o));
          }
        }
      }
      for(int t = tb; t < te; t++, tcount++) {
        // The task's metadata and column scales 2^(e_col - 7) are fetched before its
        // accumulators are complete, so their latency overlaps the task's MMAs.  The
        // scales alternate between two buffers: the readers of this buffer (two tasks
        // back) all passed the previous task's barrier below.
        const I8Task tk  = p.tasks[t];
        const int    st  = p.tslices[t];
        const int    er  = __ldg(p.a_exps + tk.a_exp + imt * MT + row);
        double*      scb = sc + (tcount & 1) * NT;
        constexpr int off = BF ? 0 : 7; // digit weights: 2^(e - 7 - 8d) (INT8), 2^e (BF16 pieces)
        if(et < NT) scb[et] = ldexp(1.0, __ldg(p.b_exps + tk.b_exp + int_ * NT + et) - off);
        // the epilogue threads agree on a timeout, so none is left in a barrier; the
        // barrier also publishes the scales
        const bool     waited = mbar_wait(tfull, tphase, p.err, 4);
        uint32_t       anyfail;
        asm volatile("{\n\t.reg .pred p, q;\n\tsetp.eq.u32 p, %1, 0;\n\t"
                     "bar.red.or.pred q, 1, %2, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
                     : "=r"(anyfail)
                     : "r"((uint32_t) waited), "n"(NE)
                     : "memory");
        if(anyfail) {
          ok = false;
          break;
        }
        tphase ^= 1;
        tc_fence_after();
        // Diagonal d carries the row factor 2^k, k = e_row - 7 - 8d.  INT8: groups of up to
        // three adjacent diagonals are combined exactly in int64,
        //   G = D_g * 2^16 + D_(g+1) * 2^8 + D_(g+2)   (|D| < 2^31, so |G| < 2^48),
        // and G * 2^k (k of the group's last diagonal) is formed without a conversion
        // instruction when k is well inside the normal range: the double whose bits are
        // ((1075 + k) << 52) + 2^51 + G equals (2^52 + 2^51 + G) * 2^k, and subtracting
        // (2^52 + 2^51) * 2^k leaves G * 2^k exactly.  One FP64 add and one FMA per group
        // instead of per diagonal; one rounding per group.  Otherwise (extreme row
        // exponents) each diagonal is converted and scaled on its own.  BF16x3: FP32
        // accumulators, exact in FP64.
        const bool   fast = !BF && er - 7 - 8 * (S - 1) >= -1000 && er - 7 <= 900;
        const double sr   = ldexp(1.0, er - off);
        if constexpr(BF) {
          // drain diagonal by diagonal; each diagonal's TMEM is released as soon as it
          // has been read, so the next task's MMAs into it can start
#pragma unroll
          for(int d = 0; d < S; d++) {
            if(d < st) {
              uint32_t       v[NH];
              const uint32_t ta = tmem + ((uint32_t) (q * 32) << 16) + d * NT + col0;
              tmem_ld_cols<NH>(ta, v);
              tmem_wait_ld();
              tc_fence_before();
              mbar_arrive(&tempty[d]);
#pragma unroll
              for(int x = 0; x < NH; x++) racc[x] = fma((double) __uint_as_float(v[x]), sr * scb[col0 + x], racc[x]);
            }
            else
              mbar_arrive(&tempty[d]);
          }
        }
        else {
          // columns per TMEM load round (sixteen warps: narrower rounds, as their threads
          // hold at most 96 registers: five of the eighteen warps share one sub-partition)
          constexpr int  CH = EW == 8 ? (NH >= 24 ? NH / 2 : NH) : (NH <= 12 ? NH : NH % 8 == 0 ? 8 : 4);
          static_assert(NH % CH == 0 && CH % 4 == 0, "drain chunking");
          const uint32_t tq = tmem + ((uint32_t) (q * 32) << 16) + col0;
#pragma unroll
          for(int g0 = 0; g0 < S; g0 += 3) {
            const int gl = S - g0 < 3 ? S - g0 : 3; // diagonals in this group
            if(g0 < st) {                           // (st is the same for every thread)
              const int     last = g0 + gl - 1;
              const int64_t hb   = ((int64_t) (1075 + er - 7 - 8 * last) << 52) + (1ll << 51);
              const double  bias = __longlong_as_double(hb);
#pragma unroll
              for(int c0 = 0; c0 < NH; c0 += CH) {
                uint32_t v0[CH], v1[CH], v2[CH];
                tmem_ld_cols<CH>(tq + g0 * NT + c0, v0);
                if(gl > 1 && g0 + 1 < st) tmem_ld_cols<CH>(tq + (g0 + 1) * NT + c0, v1);
                if(gl > 2 && g0 + 2 < st) tmem_ld_cols<CH>(tq + (g0 + 2) * NT + c0, v2);
                tmem_wait_ld();
                if(c0 + CH >= NH) { // the group's last columns are in registers: its TMEM
                  tc_fence_before(); // goes back to the MMA issuer before this chunk's math
                  for(int d = g0; d < g0 + gl; d++) mbar_arrive(&tempty[d]);
                }
                const bool has1 = gl > 1 && g0 + 1 < st, has2 = gl > 2 && g0 + 2 < st;
                if(fast) {
#pragma unroll
                  for(int x = 0; x < CH; x++) {
                    int64_t G = (int64_t) (int32_t) v0[x];
                    if(gl > 1) G = G * 256 + (has1 ? (int32_t) v1[x] : 0);
                    if(gl > 2) G = G * 256 + (has2 ? (int32_t) v2[x] : 0);
                    racc[c0 + x] = fma(__longlong_as_double(hb + G) - bias, scb[col0 + c0 + x], racc[c0 + x]);
                  }
                }
                else {
#pragma unroll
                  for(int x = 0; x < CH; x++) {
                    double t = (double) (int32_t) v0[x] * pow2i(-8 * g0);
                    if(has1) t = fma((double) (int32_t) v1[x], pow2i(-8 * (g0 + 1)), t);
                    if(has2) t = fma((double) (int32_t) v2[x], pow2i(-8 * (g0 + 2)), t);
                    racc[c0 + x] = fma(t * sr, scb[col0 + c0 + x], racc[c0 + x]);
                  }
                }
              }
            }
            else
              for(int d = g0; d < g0 + gl; d++) mbar_arrive(&tempty[d]);
          }
        }
      }
      if(!ok) break;
      if constexpr(EN) {
        // sum (C + alpha * result)^2 / D over the tile; C is read, not written.  One
        // partial sum per warp and tile (each thread's elements in a fixed order, then
        // a fixed shuffle tree), so the total does not depend on which CTA took a tile.
        double e = 0.0;
        if constexpr(xpose_fits<S, NT>()) {
          if(p.xpose) { // C contiguous along the columns: each load covers 32 / XC rows x XC columns
            double*   xb   = reinterpret_cast<double*>(smem + STAGES * STAGE + kTail) + (warp - 2) * XC * kXStride;
            const int rsub = lane / XC, csub = lane % XC;
#pragma unroll 1
            for(int x0 = 0; x0 < NH; x0 += XC) {
#pragma unroll
              for(int j = 0; j < XC; j++) xb[j * kXStride + lane] = p.alpha * racc[x0 + j];
              __syncwarp();
              const int    o  = nof[col0 + x0 + csub];
              const double dc = dco[col0 + x0 + csub];
              double       cv[XC];
#pragma unroll
              for(int rr = 0; rr < XC; rr++) { // the loads first, all in flight
                const int64_t ro = __shfl_sync(0xffffffffu, rowoff, rr * (32 / XC) + rsub);
                cv[rr]           = (ro >= 0 && o >= 0) ? __ldcs(p.C + ro + o) : 0.0;
              }
#pragma unroll
              for(int rr = 0; rr < XC; rr++) {
                const int     r  = rr * (32 / XC) + rsub;
                const int64_t ro = __shfl_sync(0xffffffffu, rowoff, r);
                const double  dr = __shfl_sync(0xffffffffu, drow, r);
                if(ro >= 0 && o >= 0) {
                  const double w = cv[rr] + xb[csub * kXStride + r];
                  e              = fma(w * w, recip_nr(dr + dc), e);
                }
              }
              __syncwarp(); // the next columns overwrite the buffer
            }
          }
        }
        if(!(xpose_fits<S, NT>() && p.xpose) && rowoff >= 0) {
          const double* crow = p.C + rowoff;
          constexpr int LB = NH % 8 == 0 ? 8 : 4; // loads in flight per batch
          static_assert(NH % LB == 0, "energy loads in whole batches of columns");
#pragma unroll
          for(int x0 = 0; x0 < NH; x0 += LB) { // a batch of loads in flight, then their sums
            double cv[LB];
#pragma unroll
            for(int j = 0; j < LB; j++) {
              const int o = nof[col0 + x0 + j];
              cv[j]       = o >= 0 ? __ldcs(crow + o) : 0.0;
            }
#pragma unroll
            for(int j = 0; j < LB; j++)
              if(nof[col0 + x0 + j] >= 0) {
                const double w = cv[j] + p.alpha * racc[x0 + j];
                e              = fma(w * w, recip_nr(drow + dco[col0 + x0 + j]), e);
              }
          }
        }
#pragma unroll
        for(int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
        if(lane == 0) p.en.part[(int64_t) it * EW + (warp - 2)] = e;
        continue;
      }
      // C (+)= alpha * result: one reduction per element (c + alpha * r, rounded once,
      // as a load-add-store would be; every element of C belongs to exactly one output
      // tile), performed at L2, so the epilogue does not wait for C's memory; a plain
      // store for an assignment (p.store).
      // A thread holds one row of the tile; when C is contiguous along the columns
      // instead, the warp passes its values through shared memory XC columns at a
      // time so that each reduction instruction covers 32 / XC rows x XC adjacent columns.
      if constexpr(xpose_fits<S, NT>()) {
        if(p.xpose) {
          static_assert(NH % XC == 0, "a warp's columns must be a multiple of the transpose width");
          double*   xb   = reinterpret_cast<double*>(smem + STAGES * STAGE + kTail) + (warp - 2) * XC * kXStride;
          const int rsub = lane / XC, csub = lane % XC;
#pragma unroll
          for(int x0 = 0; x0 < NH; x0 += XC) {
#pragma unroll
            for(int j = 0; j < XC; j++) xb[j * kXStride + lane] = p.alpha * racc[x0 + j];
            __syncwarp();
            const int o = nof[col0 + x0 + csub];
#pragma unroll
            for(int it = 0; it < XC; it++) { // rows it * (32 / XC) + rsub
              const int     r  = it * (32 / XC) + rsub;
              const int64_t ro = __shfl_sync(0xffffffffu, rowoff, r);
              if(ro >= 0 && o >= 0) {
                if(p.store) p.C[ro + o] = xb[csub * kXStride + r];
                else atomicAdd(p.C + ro + o, xb[csub * kXStride + r]);
              }
            }
            __syncwarp(); // the next columns overwrite the buffer
          }
          continue;
        }
      }
      if(rowoff >= 0) {
        double* crow = p.C + rowoff;
#pragma unroll
        for(int x = 0; x < NH; x++) {
          const int o = nof[col0 + x];
          if(o >= 0) {
            if(p.store) crow[o] = p.alpha * racc[x];
            else atomicAdd(crow + o, p.alpha * racc[x]);
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if(warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// ---------------------------------------------------------------- host side

// Blocks split by one kernel: the staged kernel (rows contiguous) or the general one,
// with their chunk table (first 8-row chunk of each block, then the total).
struct SplitSet {
  std::vector<SplitBlock> blocks;
  std::vector<int32_t>    cbegin;
  SplitBlock*             d_blocks = nullptr;
  int32_t*                d_cbegin = nullptr;
  int                     kmax     = 0;
};

// Digits of every stored, nonzero block of a read-only tensor under one operand view
// (side, digit count, tile rows, element size, the label classes' rows / K of the
// tensor's modes), kept in the context's arena while the tensor stays read-only, so
// that constant operands (the integrals) are split once instead of in every
// contraction that reads them.
struct DigitEntry final : DigitCacheEntry {
  Arena*                        arena = nullptr;
  int64_t*                      used  = nullptr; // the context's cache account
  int64_t                       bytes = 0;
  uint8_t*                      slices   = nullptr;
  int32_t*                      exps     = nullptr;
  int32_t*                      blockmax = nullptr;
  int*                          err      = nullptr;
  std::map<int64_t, SplitBlock> by_off; // element offset of a stored block -> its view here
  SplitSet                      staged, general;
  const double*                 src    = nullptr; // the tensor's packed store
  bool                          filled = false;   // digits written (stream order)
  void                          retire() override {
    if(arena) {
      arena->deallocate(slices);
      arena->deallocate(exps);
      arena->deallocate(blockmax);
    }
    if(used) *used -= bytes;
    arena = nullptr, used = nullptr, bytes = 0;
    slices = nullptr, exps = nullptr, blockmax = nullptr;
    filled = false;
  }
  ~DigitEntry() override {
    for(SplitSet* x: {&staged, &general}) {
      cudaFree(x->d_blocks);
      cudaFree(x->d_cbegin);
    }
    cudaFree(err);
    retire();
  }
};

struct I8Layout {
  int                     S = 0, NT = 0, esize = 1; // digits, output tile width, bytes per digit
  std::vector<SplitBlock> a_blocks, b_blocks;
  std::vector<int32_t>    a_cbegin, b_cbegin; // first 8-row chunk of each block, then the total
  // the blocks of each operand split by the staged kernel (rows contiguous) and by the
  // general one, each with its own chunk table
  SplitSet                a_staged, a_general, b_staged, b_general;
  // cached digits of a read-only operand (the layout then holds none of its blocks)
  std::shared_ptr<DigitEntry> a_cache, b_cache;
  std::vector<I8Task>     tasks;
  std::vector<I8TaskMeta> meta;
  std::vector<I8Item>     items;
  int64_t                 slice_bytes = 0, a_bytes = 0;
  int64_t                 nexp = 0, a_nexp = 0;
  double                  int8_ops = 0;
  double                  kc_per_item = 0; // mean 32-byte K steps of an output tile (all its tasks)
  SplitBlock*             d_ablocks = nullptr;
  SplitBlock*             d_bblocks = nullptr;
  int32_t*                d_acbegin = nullptr;
  int32_t*                d_bcbegin = nullptr;
  I8Task*                 d_tasks   = nullptr;
  I8Item*                 d_items   = nullptr;
  I8TaskMeta*             d_meta    = nullptr;
  int32_t*                d_blockmax = nullptr;
  uint8_t*                d_tslices  = nullptr;
  int*                    d_err     = nullptr;
  int*                    d_ctr     = nullptr; // tile counter of the GEMM's dynamic schedule
  int                     device    = -1;
  ~I8Layout() {
    if(device >= 0) {
      cudaSetDevice(device);
      for(SplitSet* x: {&a_staged, &a_general, &b_staged, &b_general}) {
        cudaFree(x->d_blocks);
        cudaFree(x->d_cbegin);
      }
      cudaFree(d_ablocks);
      cudaFree(d_bblocks);
      cudaFree(d_acbegin);
      cudaFree(d_bcbegin);
      cudaFree(d_tasks);
      cudaFree(d_items);
      cudaFree(d_meta);
      cudaFree(d_blockmax);
      cudaFree(d_tslices);
      cudaFree(d_err);
      cudaFree(d_ctr);
    }
  }
};

int nt_for(int S) { return S <= 6 ? 80 : 64; }

int64_t rup(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// The GEMM view of one operand block: rows = the outer labels (positions rpos, in C's
// order), K = the inner labels (positions kpos, in A's order), element strides of the
// block's row-major layout; tile_rows / kstep set the padding.
SplitBlock view_block(const int32_t* dims, int nmodes, const int8_t* rpos, int nr, const int8_t* kpos, int nk,
                      int tile_rows, int kstep) {
  int64_t str[kMaxModes];
  int64_t st = 1;
  for(int i = nmodes - 1; i >= 0; i--) {
    str[i] = st;
    st *= dims[i];
  }
  SplitBlock b{};
  b.nr   = nr;
  b.nk   = nk;
  b.rows = 1;
  for(int j = 0; j < nr; j++) {
    b.rdim[j] = dims[rpos[j]];
    b.rstr[j] = (int32_t) str[rpos[j]];
    b.rows *= b.rdim[j];
  }
  b.K = 1;
  for(int j = 0; j < nk; j++) {
    b.kdim[j] = dims[kpos[j]];
    b.kstr[j] = (int32_t) str[kpos[j]];
    b.K *= b.kdim[j];
  }
  b.kcontig = 1;
  for(int j = 0; j < nk; j++) b.kcontig &= (kpos[j] == nmodes - nk + j) ? 1 : 0;
  b.tile_rows = tile_rows;
  b.rows_pad  = (int32_t) rup(b.rows, tile_rows);
  b.K_pad     = (int32_t) rup(b.K, kstep);
  return b;
}

// Staged-kernel eligibility: K contiguous, row r at element offset r * K, and the two
// stages of one warp group (two rows each) fit in shared memory.
bool staged_ok(const SplitBlock& b, int esize) {
  if(esize != 1 || !b.kcontig) return false;
  int64_t st = b.K;
  for(int j = b.nr - 1; j >= 0; j--) {
    if(b.rstr[j] != st) return false;
    st *= b.rdim[j];
  }
  return staged_stage_bytes(b.K) * 2 + kStagedHead <= kStagedSmem;
}

void chunk_table(const std::vector<SplitBlock>& bl, std::vector<int32_t>& out) {
  out.resize(bl.size() + 1);
  int64_t n = 0;
  for(size_t i = 0; i < bl.size(); i++) {
    out[i] = (int32_t) n;
    n += bl[i].rows_pad / 8;
  }
  TB_EXPECTS(n < (1ll << 31), "too many split row groups");
  out[bl.size()] = (int32_t) n;
}

void partition_sets(const std::vector<SplitBlock>& all, int esize, SplitSet& st, SplitSet& ge) {
  for(const auto& b: all) {
    SplitSet& x = staged_ok(b, esize) ? st : ge;
    x.blocks.push_back(b);
    x.kmax = std::max(x.kmax, b.K);
  }
  chunk_table(st.blocks, st.cbegin);
  chunk_table(ge.blocks, ge.cbegin);
}

template<typename T>
void upload_vec(T*& dptr, const std::vector<T>& vec) {
  if(vec.empty()) return;
  TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&dptr), sizeof(T) * vec.size()));
  TB_CUDA(cudaMemcpy(dptr, vec.data(), sizeof(T) * vec.size(), cudaMemcpyHostToDevice));
}

// ea / eb: cached digits of a read-only A / B (their blocks are not split per launch).
std::shared_ptr<I8Layout> build_layout(const LabelClasses& lc, const WorkList& wl, int S, int NT, int esize,
                                       const std::shared_ptr<DigitEntry>& ea = nullptr,
                                       const std::shared_ptr<DigitEntry>& eb = nullptr) {
  auto L     = std::make_shared<I8Layout>();
  L->S       = S;
  L->NT      = NT;
  L->esize   = esize;
  L->a_cache = ea;
  L->b_cache = eb;
  const int kstep = KC / esize; // K elements per 32-byte MMA step
  std::map<int64_t, int> amap, bmap;
  int64_t                aexp = 0, bexp = 0, abytes = 0, bbytes = 0;
  L->tasks.resize(wl.tasks.size());
  L->meta.resize(wl.tasks.size());
  auto cached = [](const std::shared_ptr<DigitEntry>& e, int64_t off) -> const SplitBlock& {
    auto it = e->by_off.find(off);
    TB_EXPECTS(it != e->by_off.end(), "read-only operand block missing from its digit cache");
    return it->second;
  };
  for(const auto& g: wl.groups) {
    for(int t = g.task_begin; t < g.task_end; t++) {
      const DevTask& tk = wl.tasks[t];
      const SplitBlock* A = nullptr;
      const SplitBlock* B = nullptr;
      if(ea) A = &cached(ea, tk.a_off);
      else {
        auto ia = amap.find(tk.a_off);
        if(ia == amap.end()) {
          SplitBlock b = view_block(tk.adims, lc.na, lc.m_a, lc.nm, lc.k_a, lc.nk, MT, kstep);
          b.src_off    = tk.a_off;
          b.id         = (int32_t) L->a_blocks.size();
          b.dst_off    = abytes;
          b.exp_off    = (int32_t) aexp;
          abytes += (int64_t) b.rows_pad * b.K_pad * esize * S;
          aexp += b.rows_pad;
          ia = amap.emplace(tk.a_off, (int) L->a_blocks.size()).first;
          L->a_blocks.push_back(b);
        }
        A = &L->a_blocks[ia->second];
      }
      if(eb) B = &cached(eb, tk.b_off);
      else {
        auto ib = bmap.find(tk.b_off);
        if(ib == bmap.end()) {
          SplitBlock b = view_block(tk.bdims, lc.nb, lc.n_b, lc.nn, lc.k_b, lc.nk, L->NT, kstep);
          b.src_off    = tk.b_off;
          b.id         = (int32_t) L->b_blocks.size(); // rebased after the A blocks below
          b.dst_off    = bbytes;
          b.exp_off    = (int32_t) bexp;
          bbytes += (int64_t) b.rows_pad * b.K_pad * esize * S;
          bexp += b.rows_pad;
          ib = bmap.emplace(tk.b_off, (int) L->b_blocks.size()).first;
          L->b_blocks.push_back(b);
        }
        B = &L->b_blocks[ib->second];
      }
      I8Task it{};
      it.a_off    = A->dst_off;
      it.b_off    = B->dst_off; // rebased below (layout blocks)
      it.a_exp    = A->exp_off;
      it.b_exp    = B->exp_off;
      it.nkc      = A->K_pad / kstep;
      L->tasks[t] = it;
      I8TaskMeta mt{};
      mt.a_block = A->id;
      mt.b_block = B->id; // rebased below (layout blocks)
      int lk = 0;
      while((1ll << lk) < A->K) lk++;
      mt.log2k   = lk;
      L->meta[t] = mt;
    }
  }
  TB_EXPECTS(aexp + bexp < (1ll << 31), "too many split rows");
  for(auto& b: L->b_blocks) {
    b.dst_off += abytes;
    b.exp_off += (int32_t) aexp;
    b.id += (int32_t) L->a_blocks.size();
  }
  if(!eb) { // layout B blocks sit after the layout A blocks in the scratch arrays
    for(auto& m: L->meta) m.b_block += (int32_t) L->a_blocks.size();
    for(auto& t: L->tasks) {
      t.b_off += abytes;
      t.b_exp += (int32_t) aexp;
    }
  }
  L->a_bytes     = abytes;
  L->slice_bytes = abytes + bbytes;
  L->a_nexp      = aexp;
  L->nexp        = aexp + bexp;
  auto chunks    = [](const std::vector<SplitBlock>& bl, std::vector<int32_t>& out) {
    out.resize(bl.size() + 1);
    int64_t n = 0;
    for(size_t i = 0; i < bl.size(); i++) {
      out[i] = (int32_t) n;
      n += bl[i].rows_pad / 8;
    }
    out[bl.size()] = (int32_t) n;
  };
  chunks(L->a_blocks, L->a_cbegin);
  chunks(L->b_blocks, L->b_cbegin);
  partition_sets(L->a_blocks, esize, L->a_staged, L->a_general);
  partition_sets(L->b_blocks, esize, L->b_staged, L->b_general);
  // Output tiles, longest group first (every tile of a group costs the same, so
  // ordering the groups orders the tiles).  Among groups of equal work, those whose
  // first task reads the same A block (the same rows: e.g. W(a,b,c,..) = v(b,c,..) *
  // t2(a,..) for every a tile) are interleaved row tile by row tile, so the CTAs that
  // take consecutive tiles read each A tile's digits from HBM once and from L2 after.
  struct Ord {
    int64_t work, akey;
    int32_t group;
  };
  std::vector<Ord> order;
  for(size_t gi = 0; gi < wl.groups.size(); gi++) {
    const DevGroup& g = wl.groups[gi];
    if(g.task_begin == g.task_end) continue;
    int64_t work = 0;
    for(int t = g.task_begin; t < g.task_end; t++) work += L->tasks[t].nkc;
    order.push_back(Ord{work, L->tasks[g.task_begin].a_off, (int32_t) gi});
  }
  std::stable_sort(order.begin(), order.end(), [](const Ord& a, const Ord& b) {
    return a.work != b.work ? a.work > b.work : a.akey < b.akey;
  });
  auto tiles_of = [&](int32_t gi, int64_t& mts, int64_t& nts) {
    const DevGroup& g = wl.groups[gi];
    int64_t         M = 1, N = 1;
    for(int j = 0; j < lc.nm; j++) M *= g.cdims[lc.m_c[j]];
    for(int j = 0; j < lc.nn; j++) N *= g.cdims[lc.n_c[j]];
    mts = (M + MT - 1) / MT;
    nts = (N + L->NT - 1) / L->NT;
  };
  for(size_t r0 = 0; r0 < order.size();) {
    size_t r1 = r0 + 1; // groups [r0, r1): equal work, same first A block
    while(r1 < order.size() && order[r1].work == order[r0].work && order[r1].akey == order[r0].akey) r1++;
    int64_t mts = 0;
    for(size_t r = r0; r < r1; r++) {
      int64_t gm = 0, gn = 0;
      tiles_of(order[r].group, gm, gn);
      mts = std::max(mts, gm);
    }
    for(int64_t mt = 0; mt < mts; mt++)
      for(size_t r = r0; r < r1; r++) {
        int64_t gm = 0, gn = 0;
        tiles_of(order[r].group, gm, gn);
        if(mt >= gm) continue;
        for(int64_t nt = 0; nt < gn; nt++) L->items.push_back(I8Item{order[r].group, (int32_t) mt, (int32_t) nt, 0});
      }
    for(size_t r = r0; r < r1; r++) {
      int64_t gm = 0, gn = 0;
      tiles_of(order[r].group, gm, gn);
      L->int8_ops += 2.0 * MT * L->NT * kstep * order[r].work * (S * (S + 1) / 2) * (double) (gm * gn);
      L->kc_per_item += (double) order[r].work * (double) (gm * gn);
    }
    r0 = r1;
  }
  if(!L->items.empty()) L->kc_per_item /= (double) L->items.size();
  TB_CUDA(cudaGetDevice(&L->device));
  auto up = [](auto*& dptr, const auto& vec) {
    using T = std::remove_reference_t<decltype(vec[0])>;
    if(vec.empty()) return;
    TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&dptr), sizeof(T) * vec.size()));
    TB_CUDA(cudaMemcpy(dptr, vec.data(), sizeof(T) * vec.size(), cudaMemcpyHostToDevice));
  };
  up(L->d_ablocks, L->a_blocks);
  up(L->d_bblocks, L->b_blocks);
  for(SplitSet* x: {&L->a_staged, &L->a_general, &L->b_staged, &L->b_general}) {
    up(x->d_blocks, x->blocks);
    up(x->d_cbegin, x->cbegin);
  }
  up(L->d_acbegin, L->a_cbegin);
  up(L->d_bcbegin, L->b_cbegin);
  up(L->d_tasks, L->tasks);
  up(L->d_items, L->items);
  up(L->d_meta, L->meta);
  TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&L->d_blockmax),
                     sizeof(int32_t) * std::max<size_t>(1, L->a_blocks.size() + L->b_blocks.size())));
  TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&L->d_tslices), std::max<size_t>(1, L->tasks.size())));
  TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&L->d_err), sizeof(int)));
  TB_CUDA(cudaMemset(L->d_err, 0, sizeof(int)));
  TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&L->d_ctr), sizeof(int)));
  return L;
}

int sm_count() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

template<int S, int TR>
void launch_staged(const SplitSet& x, const double* src, uint8_t* slices, int32_t* exps,
                   int32_t* blockmax, int* err, cudaStream_t st) {
  const int      nblocks = (int) x.cbegin.size() - 1, nchunks = x.cbegin.back();
  const uint32_t sb      = (uint32_t) staged_stage_bytes(x.kmax);
  const int      ngroups = (int) std::min<int64_t>(kSplitMaxGroups, (kStagedSmem - kStagedHead) / (2 * (int64_t) sb));
  TB_EXPECTS(ngroups >= 1, "staged split: one group's stages must fit in shared memory");
  const size_t   smem    = kStagedHead + (size_t) 2 * ngroups * sb;
  static bool    configured[64] = {false};
  int            dev            = 0;
  TB_CUDA(cudaGetDevice(&dev));
  if(dev < 64 && !configured[dev]) {
    TB_CUDA(cudaFuncSetAttribute(k_split_staged<S, TR>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStagedSmem));
    configured[dev] = true;
  }
  const int grid = (int) std::min<int64_t>((int64_t) nchunks, sm_count()); // whole chunks per CTA
  k_split_staged<S, TR><<<grid, 32 * (1 + ngroups * kSplitGroup), smem, st>>>(
    x.d_blocks, x.d_cbegin, nblocks, nchunks, ngroups, sb, src, slices, exps, blockmax, err);
}

// Splits the blocks of one operand: the staged kernel for the blocks with contiguous
// rows, the general kernel for the rest.
template<int S, bool BF>
void split_sets(const SplitSet& staged, const SplitSet& general, const double* src, uint8_t* slices,
                int32_t* exps, int32_t* blockmax, int* err, cudaStream_t st) {
  if(!general.blocks.empty() && general.cbegin.back() > 0) {
    const int nblocks = (int) general.cbegin.size() - 1, nchunks = general.cbegin.back();
    k_split_fused<S, BF><<<std::min(nchunks, sm_count() * 8), 256, 0, st>>>(general.d_blocks, general.d_cbegin,
                                                                            nblocks, nchunks, src, slices, exps,
                                                                            blockmax);
  }
  if constexpr(!BF) {
    if(!staged.blocks.empty() && staged.cbegin.back() > 0) {
      // A tiles (128 rows) with the row count fixed at compile time, B tiles read it
      if(staged.blocks.front().tile_rows == MT) launch_staged<S, MT>(staged, src, slices, exps, blockmax, err, st);
      else launch_staged<S, 0>(staged, src, slices, exps, blockmax, err, st);
    }
  }
}

template<int S, bool BF>
void launch_split(const I8Layout& L, const WorkList& wl, const double* A, const double* B, uint8_t* slices,
                  int32_t* exps, cudaStream_t st) {
  // a read-only operand's cached digits are split once, on first use
  for(DigitEntry* e: {L.a_cache.get(), L.b_cache.get()})
    if(e && !e->filled) {
      TB_CUDA(cudaMemsetAsync(e->blockmax, 0x80, sizeof(int32_t) * std::max<size_t>(e->by_off.size(), 1), st));
      split_sets<S, BF>(e->staged, e->general, e->src, e->slices, e->exps, e->blockmax, e->err, st);
      e->filled = true;
    }
  // 0x80808080: below every exponent sum, marks blocks without a nonzero row
  TB_CUDA(cudaMemsetAsync(L.d_blockmax, 0x80, sizeof(int32_t) * (L.a_blocks.size() + L.b_blocks.size()), st));
  split_sets<S, BF>(L.a_staged, L.a_general, A, slices, exps, L.d_blockmax, L.d_err, st);
  split_sets<S, BF>(L.b_staged, L.b_general, B, slices, exps, L.d_blockmax, L.d_err, st);
  const int ng = (int) wl.groups.size();
  if constexpr(BF) { // both bf16 pieces in every task
    if(!L.tasks.empty()) TB_CUDA(cudaMemsetAsync(L.d_tslices, S, L.tasks.size(), st));
  }
  else if(ng > 0)
    k_task_slices<<<(ng + 7) / 8, 256, 0, st>>>(L.d_meta, wl.d_groups, ng,
                                                L.a_cache ? L.a_cache->blockmax : L.d_blockmax,
                                                L.b_cache ? L.b_cache->blockmax : L.d_blockmax, S, L.d_tslices);
  TB_CUDA(cudaGetLastError());
}

// Output tiles with at most this many 32-byte K steps on average (all their tasks) take
// the kernel with sixteen epilogue warps: the triples' contractions over one virtual
// index (one task of K = 250: 8 steps) or one occupied index (tasks of K = 40 and 10: 3
// steps) measured 6 % faster with them; the ladder's (tens of tasks of 18-72 steps)
// keep eight, and so does the energy gradient, which ran 1.5x slower when its
// contractions of up to 32 steps per tile took sixteen.
constexpr double kShortKSteps = 8.0;

template<int S, int NT, bool BF>
void launch_gemm(const I8Layout& L, const WorkList& wl, const LabelClasses& lc, double alpha,
                 const uint8_t* slices, const int32_t* exps, double* C, const Plan& plan, cudaStream_t st) {
  if(L.items.empty()) return;
  I8Params p;
  p.a_slices = L.a_cache ? L.a_cache->slices : slices;
  p.b_slices = L.b_cache ? L.b_cache->slices : slices;
  p.a_exps   = L.a_cache ? L.a_cache->exps : exps;
  p.b_exps   = L.b_cache ? L.b_cache->exps : exps;
  p.tasks  = L.d_tasks;
  p.groups = wl.d_groups;
  p.items  = L.d_items;
  p.nitems = (int) L.items.size();
  p.C      = C;
  p.alpha  = alpha;
  p.lc     = lc;
  p.err     = L.d_err;
  p.tslices = L.d_tslices;
  p.ctr     = L.d_ctr;
  // transposed reductions when C's last mode (stride 1) is a column label of the tile
  p.xpose = xpose_fits<S, NT>() && lc.nn > 0 && lc.n_c[lc.nn - 1] == lc.nc - 1 ? 1 : 0;
  p.store = plan.store ? 1 : 0;
  if(plan.energy) {
    p.energy = 1;
    p.en     = *plan.energy;
  }
  TB_CUDA(cudaMemsetAsync(L.d_ctr, 0, sizeof(int), st));
  const size_t smem = smem_bytes<S, NT>();
  static bool  configured[64][3] = {};
  int          dev            = 0;
  TB_CUDA(cudaGetDevice(&dev));
  // kernel: 0 the default, 1 the energy epilogue, 2 sixteen epilogue warps (a C update
  // whose tiles have little K: the epilogue, not the tensor pipe, bounds them)
  const int e = plan.energy ? 1 : (!BF && L.kc_per_item <= kShortKSteps) ? 2 : 0;
  if(dev < 64 && !configured[dev][e]) {
    if(e == 1)
      TB_CUDA(cudaFuncSetAttribute(k_contract_i8<S, NT, BF, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int) smem));
    else if(e == 2) {
      if constexpr(!BF)
        TB_CUDA(cudaFuncSetAttribute(k_contract_i8<S, NT, false, false, 16>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    }
    else TB_CUDA(cudaFuncSetAttribute(k_contract_i8<S, NT, BF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    configured[dev][e] = true;
  }
  const int grid = (int) std::min<int64_t>((int64_t) L.items.size(), sm_count());
  if(e == 1) k_contract_i8<S, NT, BF, true><<<grid, NTHREADS, smem, st>>>(p);
  else if(e == 2) {
    if constexpr(!BF) k_contract_i8<S, NT, false, false, 16><<<grid, 64 + 32 * 16, smem, st>>>(p);
  }
  else k_contract_i8<S, NT, BF><<<grid, NTHREADS, smem, st>>>(p);
  TB_CUDA(cudaGetLastError());
  if(plan.energy)
    launch_energy_final(p.en.part, (int64_t) L.items.size() * (NEPI / 32), plan.energy_scale, plan.energy_out, st);
}

template<int S, bool BF = false>
void run_s(const I8Layout& L, const WorkList& wl, const LabelClasses& lc, double alpha, const double* A,
           const double* B, double* C, uint8_t* slices, int32_t* exps, const Plan& plan, cudaStream_t st,
           cudaEvent_t* ev) {
  if(ev) TB_CUDA(cudaEventRecord(ev[0], st));
  launch_split<S, BF>(L, wl, A, B, slices, exps, st);
  if(ev) TB_CUDA(cudaEventRecord(ev[1], st));
  // output tile width: 80 columns by default for S <= 6 (S x NT <= 512 TMEM columns)
  if constexpr(S * 80 <= 512) {
    if(L.NT == 80) launch_gemm<S, 80, BF>(L, wl, lc, alpha, slices, exps, C, plan, st);
  }
  if(L.NT == 64) launch_gemm<S, 64, BF>(L, wl, lc, alpha, slices, exps, C, plan, st);
  if(L.NT == 48) launch_gemm<S, 48, BF>(L, wl, lc, alpha, slices, exps, C, plan, st);
  if(ev) TB_CUDA(cudaEventRecord(ev[2], st));
}

// Largest slice count for an error target: the truncation bound S * 2^(2 - 8S) of
// row-max x col-max x K, times 2^6 for the cancellation between that scale and the
// largest |C| seen on coupled-cluster data (O=40/V=360 ladder, balanced digits:
// S = 5 -> 6.3e-10, S = 6 -> 2.9e-12, S = 7 -> 1.4e-14 measured); smallest S meeting
// the target.
int slices_for(double err_target) {
  for(int S = 3; S <= 8; S++)
    if(S * std::ldexp(1.0, 2 - 8 * S) * 64.0 <= err_target) return S;
  return 8;
}

std::map<const WorkList*, std::shared_ptr<I8Layout>> g_layouts; // per work list, keyed by S below

// The cached digits of read-only tensor T as operand `side` (0 = A, 1 = B) of a
// contraction with the plan's label classes, for S digits, `tile_rows` rows per tile
// and esize-byte elements: every stored block the scan did not find zero, split on
// first use (launch_split) into arena memory counted against the context's cache
// budget.  Null when the budget does not allow it.
std::shared_ptr<DigitEntry> digit_entry(const Plan& plan, const Tensor* T, int side, int S, int tile_rows,
                                        int esize) {
  if(T == nullptr || plan.cache_used == nullptr || plan.arena == nullptr || !T->read_only) return nullptr;
  const LabelClasses& lc = plan.lc;
  const int8_t*       rp = side == 0 ? lc.m_a : lc.n_b;
  const int           nr = side == 0 ? lc.nm : lc.nn;
  const int8_t*       kp = side == 0 ? lc.k_a : lc.k_b;
  std::string         key = std::to_string(side) + "|" + std::to_string(S) + "|" + std::to_string(tile_rows) + "|" +
                    std::to_string(esize) + "|";
  for(int j = 0; j < nr; j++) key += std::to_string(rp[j]) + ",";
  key += "|";
  for(int j = 0; j < lc.nk; j++) key += std::to_string(kp[j]) + ",";
  auto hit = T->digit_cache.find(key);
  if(hit != T->digit_cache.end()) return std::static_pointer_cast<DigitEntry>(hit->second);
  auto                    e     = std::make_shared<DigitEntry>();
  const int               kstep = KC / esize;
  int64_t                 sbytes = 0, nexp = 0;
  std::vector<SplitBlock> all;
  std::vector<int64_t>    bid(T->nmodes);
  int32_t                 dims[kMaxModes];
  for(size_t b = 0; b < T->keys.size(); b++) {
    if(!T->zero_block.empty() && T->zero_block[b]) continue; // its tasks never run
    int64_t k = T->keys[b];
    for(int m = T->nmodes - 1; m >= 0; m--) {
      bid[m] = k % T->tis[m]->ntiles();
      k /= T->tis[m]->ntiles();
    }
    for(int m = 0; m < T->nmodes; m++) dims[m] = (int32_t) T->tis[m]->size(bid[m]);
    SplitBlock v = view_block(dims, T->nmodes, rp, nr, kp, lc.nk, tile_rows, kstep);
    v.src_off    = T->offsets[b];
    v.id         = (int32_t) all.size();
    v.dst_off    = sbytes;
    v.exp_off    = (int32_t) nexp;
    sbytes += (int64_t) v.rows_pad * v.K_pad * esize * S;
    nexp += v.rows_pad;
    TB_EXPECTS(nexp < (1ll << 31), "too many split rows");
    all.push_back(v);
    e->by_off[v.src_off] = v;
  }
  const int64_t total = sbytes + 4 * nexp + 4 * (int64_t) std::max<size_t>(all.size(), 1);
  if(*plan.cache_used + total > plan.cache_limit) return nullptr;
  e->arena    = plan.arena;
  e->slices   = static_cast<uint8_t*>(plan.arena->allocate(std::max<int64_t>(sbytes, 1)));
  e->exps     = static_cast<int32_t*>(plan.arena->allocate(4 * std::max<int64_t>(nexp, 1)));
  e->blockmax = static_cast<int32_t*>(plan.arena->allocate(4 * (int64_t) std::max<size_t>(all.size(), 1)));
  e->used     = plan.cache_used;
  e->bytes    = total;
  *e->used += total;
  TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&e->err), sizeof(int)));
  TB_CUDA(cudaMemset(e->err, 0, sizeof(int)));
  partition_sets(all, esize, e->staged, e->general);
  for(SplitSet* x: {&e->staged, &e->general}) {
    upload_vec(x->d_blocks, x->blocks);
    upload_vec(x->d_cbegin, x->cbegin);
  }
  e->src                  = T->data;
  T->digit_cache[key]     = e;
  return e;
}

} // namespace

// Split contraction, shared by the split-INT8 mode (bf = false: S balanced INT8 digits)
// and the BF16x3 mode (bf = true: two bf16 pieces, three products, FP32 accumulators).
void contract_split(Plan& plan, const WorkList& wl, double alpha, const double* A, const double* B, double* C,
                    cudaStream_t stream, bool bf) {
  const LabelClasses& lc = plan.lc;
  if(lc.nbatch > 0 || lc.nar > 0 || lc.nbr > 0 || lc.nk == 0) {
    // Hadamard / one-sided reduction labels and outer products run on the FP64 path.
    launch_contract_fp64(plan, wl, alpha, 1.0, plan.store ? 1 : 0, A, B, C, stream);
    return;
  }
  const int S     = bf ? 2 : (plan.nslices > 0 ? std::min(std::max(plan.nslices, 3), 8) : slices_for(plan.err_target));
  const int NT    = plan.tile_n > 0 ? plan.tile_n : nt_for(S);
  const int esize = bf ? 2 : 1;
  TB_EXPECTS((NT == 48 || NT == 64 || NT == 80) && S * NT <= 512,
             "split output tile width must be 48, 64 or 80 with slices x width <= 512");
  // digits of read-only operands kept across contractions (when the context allows it)
  const auto ea = digit_entry(plan, plan.cache_a, 0, S, MT, esize);
  const auto eb = digit_entry(plan, plan.cache_b, 1, S, NT, esize);
  auto&      L  = g_layouts[&wl];
  if(!L || L->S != S || L->NT != NT || L->esize != esize || L->a_cache != ea || L->b_cache != eb)
    L = build_layout(lc, wl, S, NT, esize, ea, eb);
  Scratch sc;
  sc.stream = stream;
  sc.arena  = plan.arena;
  const int64_t ebytes = sizeof(int32_t) * std::max<int64_t>(L->nexp, 1);
  auto* slices = static_cast<uint8_t*>(plan.pinned ? plan.pinned->get(L->slice_bytes) : sc.get(L->slice_bytes));
  auto* exps   = static_cast<int32_t*>(plan.pinned ? plan.pinned->get(ebytes) : sc.get(ebytes));
  cudaEvent_t  evs[3];
  cudaEvent_t* ev = nullptr;
  if(plan.profile) {
    for(auto& e: evs) TB_CUDA(cudaEventCreate(&e));
    ev = evs;
  }
  const Plan& st = plan;
  if(bf) run_s<2, true>(*L, wl, lc, alpha, A, B, C, slices, exps, st, stream, ev);
  else switch(S) {
    case 3: run_s<3>(*L, wl, lc, alpha, A, B, C, slices, exps, st, stream, ev); break;
    case 4: run_s<4>(*L, wl, lc, alpha, A, B, C, slices, exps, st, stream, ev); break;
    case 5: run_s<5>(*L, wl, lc, alpha, A, B, C, slices, exps, st, stream, ev); break;
    case 6: run_s<6>(*L, wl, lc, alpha, A, B, C, slices, exps, st, stream, ev); break;
    case 7: run_s<7>(*L, wl, lc, alpha, A, B, C, slices, exps, st, stream, ev); break;
    default: run_s<8>(*L, wl, lc, alpha, A, B, C, slices, exps, st, stream, ev); break;
  }
  if(plan.pinned) {
    plan.pinned->put(exps);
    plan.pinned->put(slices);
  }
  else {
    sc.put(exps);
    sc.put(slices);
  }
  if(ev) {
    float a = 0, b = 0;
    TB_CUDA(cudaEventSynchronize(evs[2]));
    TB_CUDA(cudaEventElapsedTime(&a, evs[0], evs[1]));
    TB_CUDA(cudaEventElapsedTime(&b, evs[1], evs[2]));
    plan.last.split_ms = a;
    plan.last.gemm_ms  = b;
    for(auto& e: evs) cudaEventDestroy(e);
  }
  plan.last.int8_ops   = L->int8_ops;
  plan.last.slices_min = S;
  plan.last.slices_max = S;
  if(plan.profile && !L->tasks.empty()) {
    // exact INT8 work of this launch: per output tile, per task, St(St+1)/2 products
    std::vector<uint8_t> ts(L->tasks.size());
    TB_CUDA(cudaMemcpyAsync(ts.data(), L->d_tslices, ts.size(), cudaMemcpyDeviceToHost, stream));
    TB_CUDA(cudaStreamSynchronize(stream));
    double ops = 0, alg = 0;
    int    smin = S, smax = 1;
    for(const auto& it: L->items) {
      const DevGroup& g = wl.groups[it.group];
      int64_t         M = 1, N = 1;
      for(int j = 0; j < lc.nm; j++) M *= g.cdims[lc.m_c[j]];
      for(int j = 0; j < lc.nn; j++) N *= g.cdims[lc.n_c[j]];
      const double rows = (double) std::min<int64_t>(MT, M - (int64_t) it.mt * MT);
      const double cols = (double) std::min<int64_t>(L->NT, N - (int64_t) it.nt * L->NT);
      for(int t = g.task_begin; t < g.task_end; t++) {
        const int st = ts[t];
        ops += 2.0 * MT * L->NT * (KC / L->esize) * L->tasks[t].nkc * (st * (st + 1) / 2);
        double K = 1;
        for(int j = 0; j < lc.nk; j++) K *= wl.tasks[t].adims[lc.k_a[j]];
        alg += 2.0 * rows * cols * K * (st * (st + 1) / 2);
        smin = std::min(smin, st);
        smax = std::max(smax, st);
      }
    }
    plan.last.int8_ops_alg = alg;
    plan.last.int8_ops   = ops;
    plan.last.slices_min = smin;
    plan.last.slices_max = smax;
  }
  plan.last.scratch_bytes = L->slice_bytes + 4 * L->nexp;
  if(plan.check_errors) {
    int h = 0;
    TB_CUDA(cudaMemcpyAsync(&h, L->d_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
    TB_CUDA(cudaStreamSynchronize(stream));
    if(h != 0) {
      cudaMemsetAsync(L->d_err, 0, sizeof(int), stream);
      fail(TB_ERR_TIMEOUT, "split-INT8 contraction: a device-side wait gave up (code " + std::to_string(h) + ")");
    }
  }
}

void forget_int8_layout(const WorkList* wl) { g_layouts.erase(wl); }

int int8_slices_for(double err_target) { return slices_for(err_target); }

void check_int8_errors(const WorkList& wl, cudaStream_t stream) {
  auto it = g_layouts.find(&wl);
  if(it == g_layouts.end() || !it->second) return;
  int h = 0;
  TB_CUDA(cudaMemcpyAsync(&h, it->second->d_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
  TB_CUDA(cudaStreamSynchronize(stream));
  if(h != 0) {
    cudaMemsetAsync(it->second->d_err, 0, sizeof(int), stream);
    fail(TB_ERR_TIMEOUT, "split-INT8 contraction: a device-side wait gave up (code " + std::to_string(h) + ")");
  }
}

void contract_int8(Plan& plan, const WorkList& wl, double alpha, const double* A, const double* B, double* C,
                   cudaStream_t stream) {
  contract_split(plan, wl, alpha, A, B, C, stream, false);
}

void contract_bf16x3(Plan& plan, const WorkList& wl, double alpha, const double* A, const double* B, double* C,
                     cudaStream_t stream) {
  contract_split(plan, wl, alpha, A, B, C, stream, true);
}

// ------------------------------------------------------------------------------
// Split-INT8 block multiply that allocates nothing (tb_block_multiply_int8_noalloc).
//
// Some callers cannot allocate device memory: an application whose device memory
// is already owned by other allocators (TAMM's RMM pool reserves 80% of the free
// memory at start-up and a framework's caching allocator keeps the rest, so a
// cudaMalloc here fails or fragments), or code that must not trigger the
// device-wide synchronisation that cudaMalloc / cudaFree can cause.  For them this
// entry point keeps all of its scratch (digit slices, exponents and the one-task
// work list) in one file-scope device array of fixed size, reserved when the
// library's device code is loaded and held by every GPU that loads it until exit.

namespace {

constexpr int64_t kNoAllocBytes = int64_t(64) << 20; // 64 MiB of scratch per GPU

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocDevices = 64;
// Device address of the array, looked up once per device (std::call_once: two host
// threads making their first call on one device do not race on the entry).  A
// cudaDeviceReset on the device would invalidate it, as it does every other device
// object of the library.
void*          g_noalloc_base[kNoAllocDevices] = {nullptr};
std::once_flag g_noalloc_once[kNoAllocDevices];

// Control words and descriptors at fixed offsets of the scratch.
constexpr int64_t kCtlErr = 0, kCtlCtr = 4, kCtlBlockMax = 8, kCtlSlices = 16, kCtlDesc = 256, kCtlItems = 1280;

struct NoAllocDesc {
  SplitBlock a, b;
  DevGroup   g;
  I8Task     task;
  I8TaskMeta meta;
  int32_t    mtiles, ntiles, nchunk_a, nchunk_b;
  int64_t    chunks_off;
};
static_assert(kCtlDesc + 2 * sizeof(SplitBlock) + sizeof(DevGroup) + sizeof(I8Task) + sizeof(I8TaskMeta) <=
                kCtlItems,
              "descriptor area overflows into the item list");

// Writes the work list and chunk tables of one block triple into the scratch and
// resets what must start from a known value (error word, block max exponents).
__global__ void k_noalloc_setup(NoAllocDesc d, unsigned char* base) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  if(tid == 0) {
    *reinterpret_cast<int*>(base + kCtlErr)              = 0;
    *reinterpret_cast<int*>(base + kCtlCtr)              = 0;
    reinterpret_cast<int32_t*>(base + kCtlBlockMax)[0]   = (int32_t) 0x80808080;
    reinterpret_cast<int32_t*>(base + kCtlBlockMax)[1]   = (int32_t) 0x80808080;
    SplitBlock* sb                                       = reinterpret_cast<SplitBlock*>(base + kCtlDesc);
    sb[0]                                                = d.a;
    sb[1]                                                = d.b;
    *reinterpret_cast<DevGroup*>(sb + 2)                 = d.g;
    *reinterpret_cast<I8Task*>(reinterpret_cast<DevGroup*>(sb + 2) + 1) = d.task;
    *reinterpret_cast<I8TaskMeta*>(reinterpret_cast<I8Task*>(reinterpret_cast<DevGroup*>(sb + 2) + 1) + 1) =
      d.meta;
  }
  I8Item* items = reinterpret_cast<I8Item*>(base + kCtlItems);
  for(int i = tid; i < d.mtiles * d.ntiles; i += nth) items[i] = I8Item{0, i / d.ntiles, i % d.ntiles, 0};
  if(tid == 0) { // one block per operand: first chunk 0, then the chunk count
    int32_t* cb = reinterpret_cast<int32_t*>(base + d.chunks_off);
    cb[0] = 0, cb[1] = d.nchunk_a, cb[2] = 0, cb[3] = d.nchunk_b;
  }
}

template<int S>
void noalloc_launch(const NoAllocDesc& d, unsigned char* base, int64_t exps_off, int64_t slices_off,
                    const LabelClasses& lc, double alpha, const double* A, const double* B, double* C,
                    cudaStream_t st) {
  constexpr int NT   = S <= 6 ? 80 : 64;
  SplitBlock*   sb   = reinterpret_cast<SplitBlock*>(base + kCtlDesc);
  DevGroup*     grp  = reinterpret_cast<DevGroup*>(sb + 2);
  I8Task*       tsk  = reinterpret_cast<I8Task*>(grp + 1);
  I8TaskMeta*   meta = reinterpret_cast<I8TaskMeta*>(tsk + 1);
  const int32_t* cb  = reinterpret_cast<const int32_t*>(base + d.chunks_off);
  int32_t*      bmax = reinterpret_cast<int32_t*>(base + kCtlBlockMax);
  uint8_t*      tsl  = base + kCtlSlices;
  int32_t*      exps = reinterpret_cast<int32_t*>(base + exps_off);
  uint8_t*      sl   = base + slices_off;
  k_noalloc_setup<<<8, 256, 0, st>>>(d, base);
  const int cap = sm_count() * 8;
  k_split_fused<S, false><<<std::min(d.nchunk_a, cap), 256, 0, st>>>(sb, cb, 1, d.nchunk_a, A, sl, exps, bmax);
  k_split_fused<S, false><<<std::min(d.nchunk_b, cap), 256, 0, st>>>(sb + 1, cb + 2, 1, d.nchunk_b, B, sl, exps, bmax);
  k_task_slices<<<1, 32, 0, st>>>(meta, grp, 1, bmax, bmax, S, tsl);
  I8Params p{};
  p.a_slices = sl;
  p.b_slices = sl;
  p.a_exps   = exps;
  p.b_exps   = exps;
  p.tasks   = tsk;
  p.groups  = grp;
  p.items   = reinterpret_cast<const I8Item*>(base + kCtlItems);
  p.nitems  = d.mtiles * d.ntiles;
  p.C       = C;
  p.alpha   = alpha;
  p.lc      = lc;
  p.err     = reinterpret_cast<int*>(base + kCtlErr);
  p.tslices = tsl;
  p.ctr     = reinterpret_cast<int*>(base + kCtlCtr);
  // transposed reductions when C's last mode is a column label, as the allocating path
  p.xpose = xpose_fits<S, NT>() && lc.nn > 0 && lc.n_c[lc.nn - 1] == lc.nc - 1 ? 1 : 0;
  const size_t smem = smem_bytes<S, NT>();
  TB_CUDA(cudaFuncSetAttribute(k_contract_i8<S, NT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
  k_contract_i8<S, NT, false><<<std::min(p.nitems, sm_count()), NTHREADS, smem, st>>>(p);
  TB_CUDA(cudaGetLastError());
}

} // namespace

} // namespace tb

extern "C" int tb_block_multiply_int8_noalloc(double alpha, const double* a, const int64_t* adims,
                                              const int* alabels, int na, const double* b,
                                              const int64_t* bdims, const int* blabels, int nb,
                                              double* c, const int64_t* cdims, const int* clabels,
                                              int nc, int nslices, void* stream) {
  using namespace tb;
  try {
    TB_EXPECTS(a != nullptr && b != nullptr && c != nullptr, "a, b and c must be non-null");
    TB_EXPECTS((na == 0 || (adims && alabels)) && (nb == 0 || (bdims && blabels)) && (nc == 0 || (cdims && clabels)),
               "dims/labels arrays must be given for every non-scalar operand");
    TB_EXPECTS(nslices == 0 || (nslices >= 3 && nslices <= 8), "nslices must be 0 (target 1e-11) or 3..8");
    {
      // the call drains the stream to read its status back: refused before any work
      // is enqueued while the stream is capturing, so the capture itself stays valid
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      TB_CUDA(cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cs));
      TB_EXPECTS(cs == cudaStreamCaptureStatusNone,
                 "tb_block_multiply_int8_noalloc cannot be captured into a CUDA graph (it synchronises its stream)");
    }
    const LabelClasses lc = classify(clabels, nc, alabels, na, blabels, nb);
    if(lc.nbatch > 0 || lc.nar > 0 || lc.nbr > 0 || lc.nk == 0)
      fail(TB_ERR_NOT_IMPLEMENTED, "the allocation-free split-INT8 entry point takes plain contractions only "
                                   "(no Hadamard, one-sided reduction or outer-product labels)");
    for(int i = 0; i < na; i++) TB_EXPECTS(adims[i] > 0 && adims[i] < (1 << 30), "block extent out of range");
    for(int i = 0; i < nb; i++) TB_EXPECTS(bdims[i] > 0 && bdims[i] < (1 << 30), "block extent out of range");
    for(int i = 0; i < nc; i++) TB_EXPECTS(cdims[i] > 0 && cdims[i] < (1 << 30), "block extent out of range");
    const int S  = nslices > 0 ? nslices : slices_for(1e-11);
    const int NT = S <= 6 ? 80 : 64;

    // block geometry, the same views the allocating path builds (build_layout)
    int64_t astr[kMaxModes], bstr[kMaxModes];
    {
      int64_t s = 1;
      for(int i = na - 1; i >= 0; i--) {
        astr[i] = s;
        s *= adims[i];
      }
      s = 1;
      for(int i = nb - 1; i >= 0; i--) {
        bstr[i] = s;
        s *= bdims[i];
      }
    }
    NoAllocDesc d{};
    int64_t     M = 1, N = 1, K = 1;
    for(int j = 0; j < lc.nm; j++) {
      TB_EXPECTS(cdims[lc.m_c[j]] == adims[lc.m_a[j]], "A-outer label extents differ (C vs A)");
      d.a.rdim[j] = (int32_t) adims[lc.m_a[j]];
      d.a.rstr[j] = (int32_t) astr[lc.m_a[j]];
      M *= adims[lc.m_a[j]];
    }
    for(int j = 0; j < lc.nn; j++) {
      TB_EXPECTS(cdims[lc.n_c[j]] == bdims[lc.n_b[j]], "B-outer label extents differ (C vs B)");
      d.b.rdim[j] = (int32_t) bdims[lc.n_b[j]];
      d.b.rstr[j] = (int32_t) bstr[lc.n_b[j]];
      N *= bdims[lc.n_b[j]];
    }
    for(int j = 0; j < lc.nk; j++) {
      TB_EXPECTS(adims[lc.k_a[j]] == bdims[lc.k_b[j]], "inner label extents differ (A vs B)");
      d.a.kdim[j] = d.b.kdim[j] = (int32_t) adims[lc.k_a[j]];
      d.a.kstr[j] = (int32_t) astr[lc.k_a[j]];
      d.b.kstr[j] = (int32_t) bstr[lc.k_b[j]];
      K *= adims[lc.k_a[j]];
    }
    TB_EXPECTS(M * K < (1ll << 31) && N * K < (1ll << 31) && M * N < (1ll << 31),
               "a single block must hold fewer than 2^31 elements");
    const int64_t Mp = rup(M, MT), Np = rup(N, NT), Kp = rup(K, KC);
    const int64_t abytes = S * Mp * Kp, bbytes = S * Np * Kp;
    const int64_t mtiles = Mp / MT, ntiles = Np / NT;
    const int64_t chunks_off = rup(kCtlItems + 16 * mtiles * ntiles, 256);
    const int64_t exps_off   = rup(chunks_off + 16, 256);
    const int64_t sl_off     = rup(exps_off + 4 * (Mp + Np), 256);
    const int64_t need       = sl_off + abytes + bbytes;
    if(need > kNoAllocBytes)
      fail(TB_ERR_INVALID, "tb_block_multiply_int8_noalloc: this block triple needs " + std::to_string(need) +
                             " bytes of scratch; the static scratch holds " + std::to_string(kNoAllocBytes) +
                             " bytes (64 MiB)");

    d.a.src_off = 0;
    d.a.dst_off = 0;
    d.a.exp_off = 0;
    d.a.id      = 0;
    d.a.rows    = (int32_t) M;
    d.a.K       = (int32_t) K;
    d.a.rows_pad  = (int32_t) Mp;
    d.a.K_pad     = (int32_t) Kp;
    d.a.tile_rows = MT;
    d.a.nr        = lc.nm;
    d.a.nk        = lc.nk;
    d.a.kcontig   = 1;
    for(int j = 0; j < lc.nk; j++) d.a.kcontig &= (lc.k_a[j] == na - lc.nk + j) ? 1 : 0;
    d.b.src_off   = 0;
    d.b.dst_off   = abytes;
    d.b.exp_off   = (int32_t) Mp;
    d.b.id        = 1;
    d.b.rows      = (int32_t) N;
    d.b.K         = (int32_t) K;
    d.b.rows_pad  = (int32_t) Np;
    d.b.K_pad     = (int32_t) Kp;
    d.b.tile_rows = NT;
    d.b.nr        = lc.nn;
    d.b.nk        = lc.nk;
    d.b.kcontig   = 1;
    for(int j = 0; j < lc.nk; j++) d.b.kcontig &= (lc.k_b[j] == nb - lc.nk + j) ? 1 : 0;
    d.g.c_off      = 0;
    d.g.task_begin = 0;
    d.g.task_end   = 1;
    for(int i = 0; i < nc; i++) d.g.cdims[i] = (int32_t) cdims[i];
    d.task.a_off = 0;
    d.task.b_off = abytes;
    d.task.a_exp = 0;
    d.task.b_exp = (int32_t) Mp;
    d.task.nkc   = (int32_t) (Kp / KC);
    d.meta.a_block = 0;
    d.meta.b_block = 1;
    int lk = 0;
    while((1ll << lk) < K) lk++;
    d.meta.log2k  = lk;
    d.mtiles      = (int32_t) mtiles;
    d.ntiles      = (int32_t) ntiles;
    d.nchunk_a    = (int32_t) (Mp / 8);
    d.nchunk_b    = (int32_t) (Np / 8);
    d.chunks_off  = chunks_off;

    // set-up once per device, with that device current: the device address of the
    // static scratch (its host-side name is only a stand-in, not a device address)
    int dev = 0;
    TB_CUDA(cudaGetDevice(&dev));
    TB_EXPECTS(dev >= 0 && dev < kNoAllocDevices, "device index out of range");
    std::call_once(g_noalloc_once[dev], [dev] {
      void* ptr = nullptr;
      TB_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch)); // throws: the flag stays unset
      g_noalloc_base[dev] = ptr;
    });
    auto*      base = static_cast<unsigned char*>(g_noalloc_base[dev]);
    const auto st   = static_cast<cudaStream_t>(stream);
    switch(S) {
      case 3: noalloc_launch<3>(d, base, exps_off, sl_off, lc, alpha, a, b, c, st); break;
      case 4: noalloc_launch<4>(d, base, exps_off, sl_off, lc, alpha, a, b, c, st); break;
      case 5: noalloc_launch<5>(d, base, exps_off, sl_off, lc, alpha, a, b, c, st); break;
      case 6: noalloc_launch<6>(d, base, exps_off, sl_off, lc, alpha, a, b, c, st); break;
      case 7: noalloc_launch<7>(d, base, exps_off, sl_off, lc, alpha, a, b, c, st); break;
      default: noalloc_launch<8>(d, base, exps_off, sl_off, lc, alpha, a, b, c, st); break;
    }
    int h = 0;
    TB_CUDA(cudaMemcpyAsync(&h, base + kCtlErr, sizeof(int), cudaMemcpyDeviceToHost, st));
    TB_CUDA(cudaStreamSynchronize(st));
    if(h != 0) fail(TB_ERR_TIMEOUT, "split-INT8 contraction: a device-side wait gave up (code " + std::to_string(h) + ")");
  } catch(const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch(const std::exception& e) {
    set_last_error(e.what());
    return TB_ERR_INVALID;
  }
  return TB_OK;
}
