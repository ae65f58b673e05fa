// Grouped FP64 block contraction on the FP64 tensor cores (DMMA, mma.sync m16n8k8 f64).
//
// One launch runs a whole MultOp::execute_bufacc (src/tamm/multop.hpp:576-893): every
// CTA owns one 128x64 tile of one output block (a "group") and loops over the
// group's (A block, B block) tasks — the admitted reduction tiles — and, inside each
// task, over the A-only x B-only reduction steps and the K chunks, accumulating in
// registers.  Operands are gathered straight from the block store with the label
// permutation folded into per-row / per-k offset tables (no Ainter/Binter copies as in
// kernels::block_multiply's transpose_inputs, multiply.hpp:159-194), staged through a
// 4-deep cp.async pipeline, and the result is written once into C in C's own label
// order (transpose_output, multiply.hpp:196-210, fused into the epilogue).
#include "tb_internal.hpp"

#include <algorithm>

namespace tb {
namespace {

constexpr int BM = 128, BK = 32, STAGES = 2, NSLOT = STAGES + 1, NTHREADS = 256;
// output tile width BN: 64, or 80 where that pads the work list's output blocks less

// Shared-memory tiles are stored unpadded with the column XOR-swizzled by the row's two
// low bits (in units of 4 doubles), so that the DMMA fragment loads (8 rows x 4 columns per
// half warp) hit 16 distinct bank pairs.  Dropping the padding lets 4 stages fit at 2 CTAs
// per SM.
__device__ __forceinline__ int swz(int row, int col) { return col ^ ((row & 3) << 2); }

struct TaskInfo {
  int64_t a_blk, b_blk; // block offset + batch offset, elements
  int32_t K, AR, BR, ARBR;
  int32_t kdim[kMaxClass], kstrA[kMaxClass], kstrB[kMaxClass];
  int32_t ardim[kMaxClass], arstrA[kMaxClass];
  int32_t brdim[kMaxClass], brstrB[kMaxClass];
  int32_t mstrA[kMaxClass], nstrB[kMaxClass];
};

struct ChunkDesc {
  int64_t a_base, b_base;
  int32_t valid, buf, kvalid, first_step;
  int32_t kA[BK], kB[BK];
};

template<int BN>
struct Smem {
  double    As[STAGES][BM][BK]; // [m][k ^ swz]
  double    Bs[STAGES][BK][BN]; // [k][n ^ swz]
  int32_t   rowA[2][BM];
  int32_t   colB[2][BN];
  int32_t   rowC[BM];
  int32_t   colC[BN];
  double    rowD[BM]; // energy epilogue: the rows' and columns' parts of the denominators
  double    colD[BN];
  // the output block's geometry, worked out by one thread: extents and C strides of the
  // row / column labels, batch indices of the tile, C offset of its batch
  int32_t   gmdim[kMaxClass], gmstr[kMaxClass], gndim[kMaxClass], gnstr[kMaxClass], gbidx[kMaxClass];
  int32_t   gM, gN;
  int64_t   gcbase;
  TaskInfo  ti[2];
  ChunkDesc desc[NSLOT];
};

// two CTAs per SM (228 KB of shared memory, 1 KB of it reserved per CTA)
static_assert(2 * (sizeof(Smem<80>) + 1024) <= 228 * 1024, "two FP64 CTAs per SM");

struct Params {
  LabelClasses    lc;
  const double*   A;
  const double*   B;
  double*         C;
  const DevGroup* groups;
  const DevTask*  tasks;
  const DevItem*  items;
  double          alpha, beta;
  int             is_assign;
  int             energy = 0; // sum (C + alpha * acc)^2 / D into en.part, C unchanged
  EnergyArgs      en;
};

__device__ __forceinline__ void cp_async8(uint32_t saddr, const void* gmem, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template<int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// D(16x8) += A(16x8) * B(8x8) in FP64.  Fragments (g = lane / 4, t = lane % 4):
// a = {A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4]}, b = {B[t][g], B[t+4][g]},
// c = {C[g][2t], C[g][2t+1], C[g+8][2t], C[g+8][2t+1]}.
__device__ __forceinline__ void dmma16(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
               "{%8,%9}, {%0,%1,%2,%3};\n"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Row-major strides of a block with `n` modes.
__device__ __forceinline__ void strides_of(const int32_t* dims, int n, int64_t* str) {
  int64_t s = 1;
  for(int i = n - 1; i >= 0; i--) {
    str[i] = s;
    s *= dims[i];
  }
}

// Offset of linear index x decomposed over dims[0..n) (last fastest) with strides.
__device__ __forceinline__ int32_t decompose(int32_t x, int n, const int32_t* dims,
                                             const int32_t* str) {
  int32_t off = 0;
  for(int j = n - 1; j >= 0; j--) {
    int32_t d = dims[j];
    int32_t q = x / d;
    off += (x - q * d) * str[j];
    x = q;
  }
  return off;
}

template<int BN>
__global__ void __launch_bounds__(NTHREADS, 2) k_contract_fp64(const Params p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<BN>&           s   = *reinterpret_cast<Smem<BN>*>(smem_raw);
  const LabelClasses& lc  = p.lc;
  const int           tid = threadIdx.x;
  const DevItem       it  = p.items[blockIdx.x];
  const DevGroup      g   = p.groups[it.group];
  const int           tb  = g.task_begin, te = g.task_end;

  // ---- output block geometry (uniform): one thread works it out into shared memory
  // (per-thread copies indexed by runtime label positions would live in local memory) ----
  if(tid == 0) {
    int64_t cstr[kMaxModes];
    strides_of(g.cdims, lc.nc, cstr);
    int32_t M = 1, N = 1;
    for(int j = 0; j < lc.nm; j++) {
      s.gmdim[j] = g.cdims[lc.m_c[j]];
      s.gmstr[j] = (int32_t) cstr[lc.m_c[j]];
      M *= s.gmdim[j];
    }
    for(int j = 0; j < lc.nn; j++) {
      s.gndim[j] = g.cdims[lc.n_c[j]];
      s.gnstr[j] = (int32_t) cstr[lc.n_c[j]];
      N *= s.gndim[j];
    }
    int32_t x  = it.batch;
    int64_t cb = g.c_off;
    for(int j = lc.nbatch - 1; j >= 0; j--) {
      const int32_t d = g.cdims[lc.batch_c[j]];
      s.gbidx[j]      = x % d;
      x /= d;
      cb += s.gbidx[j] * cstr[lc.batch_c[j]];
    }
    s.gM     = M;
    s.gN     = N;
    s.gcbase = cb;
  }
  __syncthreads();
  const int32_t Mtot = s.gM, Ntot = s.gN;
  const int64_t c_base = s.gcbase;
  for(int m = tid; m < BM; m += NTHREADS)
    s.rowC[m] = (it.m0 + m < Mtot) ? decompose(it.m0 + m, lc.nm, s.gmdim, s.gmstr) : 0;
  for(int n = tid; n < BN; n += NTHREADS)
    s.colC[n] = (it.n0 + n < Ntot) ? decompose(it.n0 + n, lc.nn, s.gndim, s.gnstr) : 0;
  if(p.energy) { // batch labels' part folded into the rows'
    const int32_t* es = p.en.estart + (int64_t) it.group * lc.nc;
    double         db = 0.0;
    for(int j = 0; j < lc.nbatch; j++)
      db += p.en.sg[lc.batch_c[j]] * __ldg(p.en.eps + es[lc.batch_c[j]] + s.gbidx[j]);
    for(int m = tid; m < BM; m += NTHREADS)
      s.rowD[m] = (it.m0 + m < Mtot) ? db + energy_part(it.m0 + m, lc.nm, s.gmdim, lc.m_c, p.en, es) : 0.0;
    for(int n = tid; n < BN; n += NTHREADS)
      s.colD[n] = (it.n0 + n < Ntot) ? energy_part(it.n0 + n, lc.nn, s.gndim, lc.n_c, p.en, es) : 1.0;
  }

  // ---- chunk iterator over (task, reduction step, k0), uniform across the CTA ----
  int  cur_t = tb, cur_s = 0, cur_k0 = 0, cur_K = 0, cur_ARBR = 0, cur_BR = 1;
  bool started = false;

  auto prepare = [&](int q) {
    bool new_task = false;
    if(!started) {
      started  = true;
      new_task = true;
    }
    else if(cur_t < te) {
      cur_k0 += BK;
      if(cur_k0 >= cur_K) {
        cur_k0 = 0;
        if(++cur_s >= cur_ARBR) {
          cur_s = 0;
          ++cur_t;
          new_task = true;
        }
      }
    }
    ChunkDesc& d = s.desc[q % NSLOT];
    if(cur_t >= te) {
      if(tid == 0) d.valid = 0;
      return;
    }
    const int buf = (cur_t - tb) & 1;
    TaskInfo& ti  = s.ti[buf];
    if(new_task) {
      if(tid == 0) {
        const DevTask tk = p.tasks[cur_t];
        int64_t       astr[kMaxModes], bstr[kMaxModes];
        strides_of(tk.adims, lc.na, astr);
        strides_of(tk.bdims, lc.nb, bstr);
        ti.K = 1;
        for(int j = 0; j < lc.nk; j++) {
          ti.kdim[j]  = tk.adims[lc.k_a[j]];
          ti.kstrA[j] = (int32_t) astr[lc.k_a[j]];
          ti.kstrB[j] = (int32_t) bstr[lc.k_b[j]];
          ti.K *= ti.kdim[j];
        }
        ti.AR = 1;
        for(int j = 0; j < lc.nar; j++) {
          ti.ardim[j]  = tk.adims[lc.ar_a[j]];
          ti.arstrA[j] = (int32_t) astr[lc.ar_a[j]];
          ti.AR *= ti.ardim[j];
        }
        ti.BR = 1;
        for(int j = 0; j < lc.nbr; j++) {
          ti.brdim[j]  = tk.bdims[lc.br_b[j]];
          ti.brstrB[j] = (int32_t) bstr[lc.br_b[j]];
          ti.BR *= ti.brdim[j];
        }
        ti.ARBR = ti.AR * ti.BR;
        for(int j = 0; j < lc.nm; j++) ti.mstrA[j] = (int32_t) astr[lc.m_a[j]];
        for(int j = 0; j < lc.nn; j++) ti.nstrB[j] = (int32_t) bstr[lc.n_b[j]];
        int64_t ab = tk.a_off, bb = tk.b_off;
        for(int j = 0; j < lc.nbatch; j++) {
          ab += s.gbidx[j] * astr[lc.batch_a[j]];
          bb += s.gbidx[j] * bstr[lc.batch_b[j]];
        }
        ti.a_blk = ab;
        ti.b_blk = bb;
      }
      __syncthreads();
      cur_K    = ti.K;
      cur_ARBR = ti.ARBR;
      cur_BR   = ti.BR;
      for(int m = tid; m < BM; m += NTHREADS)
        s.rowA[buf][m] = (it.m0 + m < Mtot) ? decompose(it.m0 + m, lc.nm, s.gmdim, ti.mstrA) : 0;
      for(int n = tid; n < BN; n += NTHREADS)
        s.colB[buf][n] = (it.n0 + n < Ntot) ? decompose(it.n0 + n, lc.nn, s.gndim, ti.nstrB) : 0;
    }
    if(tid == 0) {
      const int ar = cur_s / cur_BR, br = cur_s - (cur_s / cur_BR) * cur_BR;
      d.a_base     = ti.a_blk + decompose(ar, lc.nar, ti.ardim, ti.arstrA);
      d.b_base     = ti.b_blk + decompose(br, lc.nbr, ti.brdim, ti.brstrB);
      d.valid      = 1;
      d.buf        = buf;
      d.kvalid     = min(BK, cur_K - cur_k0);
      d.first_step = (cur_s > 0 && cur_k0 == 0) ? 1 : 0;
    }
    if(tid < BK) {
      const int k = cur_k0 + tid;
      d.kA[tid]   = (k < cur_K) ? decompose(k, lc.nk, ti.kdim, ti.kstrA) : 0;
    }
    else if(tid < 2 * BK) {
      const int k     = cur_k0 + tid - BK;
      d.kB[tid - BK] = (k < cur_K) ? decompose(k, lc.nk, ti.kdim, ti.kstrB) : 0;
    }
  };

  // Per-thread constants of the gather.  With K contiguous in an operand each thread
  // keeps one k column and walks rows; otherwise it keeps one row (column) and walks k,
  // so that consecutive threads read consecutive addresses either way.  The row / column
  // / k offset tables hold 0 past the block's edge, so every source address stays inside
  // the task's block; out-of-range elements are zero-filled (source size 0).
  const bool     a_kfast = lc.a_contig == 1, b_kfast = lc.b_contig == 1;
  const int      a_fix = a_kfast ? tid % BK : tid % BM, a_walk0 = a_kfast ? tid / BK : tid / BM;
  const int      b_fix = b_kfast ? tid % BK : tid % BN, b_walk0 = b_kfast ? tid / BK : tid / BN;
  const int      m_lim = Mtot - it.m0, n_lim = Ntot - it.n0;
  const uint32_t sA0   = static_cast<uint32_t>(__cvta_generic_to_shared(&s.As[0][0][0]));
  const uint32_t sB0   = static_cast<uint32_t>(__cvta_generic_to_shared(&s.Bs[0][0][0]));

  auto issue = [&](int q) {
    const ChunkDesc& d = s.desc[q % NSLOT];
    if(!d.valid) return;
    const int      stage = q % STAGES, buf = d.buf, kvalid = d.kvalid;
    const uint32_t sA    = sA0 + stage * (BM * BK * 8), sB = sB0 + stage * (BK * BN * 8);
    constexpr int  EA = (BM * BK) / NTHREADS, EB = (BK * BN) / NTHREADS;
    if(a_kfast) { // thread: k = a_fix, rows a_walk0 + e * (NTHREADS / BK)
      const bool    kok = a_fix < kvalid;
      const double* src = p.A + d.a_base + d.kA[a_fix];
#pragma unroll
      for(int e = 0; e < EA; e++) {
        const int  m  = a_walk0 + e * (NTHREADS / BK);
        const bool ok = kok && m < m_lim;
        cp_async8(sA + (m * BK + swz(m, a_fix)) * 8, src + s.rowA[buf][m], ok ? 8 : 0);
      }
    }
    else { // thread: row = a_fix, k = a_walk0 + e * (NTHREADS / BM)
      const bool    mok = a_fix < m_lim;
      const double* src = p.A + d.a_base + s.rowA[buf][a_fix];
#pragma unroll
      for(int e = 0; e < EA; e++) {
        const int  kk = a_walk0 + e * (NTHREADS / BM);
        const bool ok = mok && kk < kvalid;
        cp_async8(sA + (a_fix * BK + swz(a_fix, kk)) * 8, src + d.kA[kk], ok ? 8 : 0);
      }
    }
    if(b_kfast) { // thread: k = b_fix, columns b_walk0 + e * (NTHREADS / BK)
      const bool    kok = b_fix < kvalid;
      const double* src = p.B + d.b_base + d.kB[b_fix];
#pragma unroll
      for(int e = 0; e < EB; e++) {
        const int  n  = b_walk0 + e * (NTHREADS / BK);
        const bool ok = kok && n < n_lim;
        cp_async8(sB + (b_fix * BN + swz(b_fix, n)) * 8, src + s.colB[buf][n], ok ? 8 : 0);
      }
    }
    else if constexpr(NTHREADS % BN == 0) { // thread: column = b_fix, k = b_walk0 + e * (NTHREADS / BN)
      const bool    nok = b_fix < n_lim;
      const double* src = p.B + d.b_base + s.colB[buf][b_fix];
#pragma unroll
      for(int e = 0; e < EB; e++) {
        const int  kk = b_walk0 + e * (NTHREADS / BN);
        const bool ok = nok && kk < kvalid;
        cp_async8(sB + (kk * BN + swz(kk, b_fix)) * 8, src + d.kB[kk], ok ? 8 : 0);
      }
    }
    else { // a width that does not divide the thread count: P = NTHREADS / BN rows of BN
           // columns per pass on the first P * BN threads, each keeping its column
      constexpr int P = NTHREADS / BN, NE = (BK + P - 1) / P;
      if(tid < P * BN) {
        const int     n   = tid % BN, k0 = tid / BN;
        const bool    nok = n < n_lim;
        const double* src = p.B + d.b_base + s.colB[buf][n];
#pragma unroll
        for(int e = 0; e < NE; e++) {
          const int kk = k0 + e * P;
          if(kk < BK) cp_async8(sB + (kk * BN + swz(kk, n)) * 8, src + d.kB[kk], nok && kk < kvalid ? 8 : 0);
        }
      }
    }
  };

  // each warp owns a 32 x BN/2 piece of the tile: 2 (m16) x NJ (n8) DMMA tiles
  constexpr int NJ = BN / 16;
  static_assert(BN % 16 == 0, "tile width must be a multiple of 16");
  const int warp = tid >> 5, lane = tid & 31, lg = lane >> 2, lt = lane & 3;
  const int wm = (warp & 3) * 32, wn = (warp >> 2) * (BN / 2);
  double    acc[2][NJ][4];
#pragma unroll
  for(int i = 0; i < 2; i++)
#pragma unroll
    for(int j = 0; j < NJ; j++)
#pragma unroll
      for(int h = 0; h < 4; h++) acc[i][j][h] = 0.0;

  // ---- prologue: chunks 0..STAGES-2 in flight, chunk STAGES-1 prepared ----
  prepare(0);
  __syncthreads();
#pragma unroll 1
  for(int q = 0; q < STAGES - 1; q++) {
    issue(q);
    cp_async_commit();
    prepare(q + 1);
    __syncthreads();
  }

#pragma unroll 1
  for(int q = 0;; q++) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const ChunkDesc& dq = s.desc[q % NSLOT];
    if(!dq.valid) break;
    const bool scale_acc = dq.first_step != 0;
    issue(q + STAGES - 1);
    cp_async_commit();
    prepare(q + STAGES);
    if(scale_acc) { // beta chaining of A-only x B-only reduction steps (gemm_wrapper)
#pragma unroll
      for(int i = 0; i < 2; i++)
#pragma unroll
        for(int j = 0; j < NJ; j++)
#pragma unroll
          for(int h = 0; h < 4; h++) acc[i][j][h] *= p.beta;
    }
    const int stage = q % STAGES;
#pragma unroll
    for(int k8 = 0; k8 < BK; k8 += 8) {
      double a[2][4];
#pragma unroll
      for(int i = 0; i < 2; i++) {
        const int r = wm + 16 * i + lg;
        a[i][0]     = s.As[stage][r][swz(r, k8 + lt)];
        a[i][1]     = s.As[stage][r + 8][swz(r, k8 + lt)];
        a[i][2]     = s.As[stage][r][swz(r, k8 + lt + 4)];
        a[i][3]     = s.As[stage][r + 8][swz(r, k8 + lt + 4)];
      }
#pragma unroll
      for(int j = 0; j < NJ; j++) { // one B fragment live at a time
        double b[2];
        b[0] = s.Bs[stage][k8 + lt][swz(lt, wn + 8 * j + lg)];
        b[1] = s.Bs[stage][k8 + lt + 4][swz(lt, wn + 8 * j + lg)];
        dmma16(acc[0][j], a[0], b);
        dmma16(acc[1][j], a[1], b);
      }
    }
  }
  cp_async_wait<0>();

  if(p.energy) { // sum (C + alpha * acc)^2 / D over the tile, C unchanged; a partial per warp
    double e = 0.0;
#pragma unroll
    for(int i = 0; i < 2; i++) {
#pragma unroll
      for(int hr = 0; hr < 2; hr++) {
        const int m = wm + 16 * i + 8 * hr + lg;
        if(it.m0 + m >= Mtot) continue;
        const int64_t rbase = c_base + s.rowC[m];
        const double  dr    = s.rowD[m];
#pragma unroll
        for(int j = 0; j < NJ; j++) {
#pragma unroll
          for(int h = 0; h < 2; h++) {
            const int n = wn + 8 * j + 2 * lt + h;
            if(it.n0 + n >= Ntot) continue;
            const double w = __ldcs(p.C + rbase + s.colC[n]) + p.alpha * acc[i][j][2 * hr + h];
            e              = fma(w * w, recip_nr(dr + s.colD[n]), e);
          }
        }
      }
    }
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if((tid & 31) == 0) p.en.part[(int64_t) blockIdx.x * (NTHREADS / 32) + (tid >> 5)] = e;
    return;
  }
  // ---- epilogue: C (=|+=) alpha * acc in C's own layout ----
#pragma unroll
  for(int i = 0; i < 2; i++) {
#pragma unroll
    for(int hr = 0; hr < 2; hr++) {
      const int m = wm + 16 * i + 8 * hr + lg;
      if(it.m0 + m >= Mtot) continue;
      const int64_t rbase = c_base + s.rowC[m];
#pragma unroll
      for(int j = 0; j < NJ; j++) {
#pragma unroll
        for(int h = 0; h < 2; h++) {
          const int n = wn + 8 * j + 2 * lt + h;
          if(it.n0 + n >= Ntot) continue;
          double*      cp = p.C + rbase + s.colC[n];
          const double v  = p.alpha * acc[i][j][2 * hr + h];
          *cp             = p.is_assign ? v : *cp + v;
        }
      }
    }
  }
}

} // namespace

static void build_items_fp64(const LabelClasses& lc, const WorkList& wl);

template<int BN>
static void launch_k(const Params& p, unsigned nitems, cudaStream_t stream) {
  const size_t smem = sizeof(Smem<BN>);
  static bool  configured[64] = {false};
  int          dev            = 0;
  TB_CUDA(cudaGetDevice(&dev));
  if(dev < 64 && !configured[dev]) {
    TB_CUDA(cudaFuncSetAttribute(k_contract_fp64<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    configured[dev] = true;
  }
  k_contract_fp64<BN><<<nitems, NTHREADS, smem, stream>>>(p);
  TB_CUDA(cudaGetLastError());
}

void launch_contract_fp64(const Plan& plan, const WorkList& wl, double alpha, double beta,
                          int is_assign, const double* A, const double* B, double* C,
                          cudaStream_t stream) {
  if(!wl.items_built) build_items_fp64(plan.lc, wl);
  if(wl.items_fp64.empty()) return;
  Params p;
  p.lc        = plan.lc;
  p.A         = A;
  p.B         = B;
  p.C         = C;
  p.groups    = wl.d_groups;
  p.tasks     = wl.d_tasks;
  p.items     = wl.d_items;
  p.alpha     = alpha;
  p.beta      = beta;
  p.is_assign = is_assign;
  if(plan.energy) {
    TB_EXPECTS(!is_assign && beta == 1.0, "energy epilogue of an assignment");
    p.energy = 1;
    p.en     = *plan.energy;
  }
  const int64_t nitems = (int64_t) wl.items_fp64.size();
  TB_EXPECTS(nitems < (1ll << 31), "work list too large");
  if(wl.items_bn == 80) launch_k<80>(p, (unsigned) nitems, stream);
  else launch_k<64>(p, (unsigned) nitems, stream);
  if(plan.energy) launch_energy_final(p.en.part, nitems * (NTHREADS / 32), plan.energy_scale, plan.energy_out, stream);
}

// Work items of the FP64 kernel: one per (group, batch index, 128-row tile, BN-column
// tile), longest group first so the hardware block scheduler balances uneven groups
// (every tile of a group costs the same, so ordering the groups orders the tiles).
// BN is 80 where that pads the output columns of the work list less than 64 does
// (N = 400 or 80, say), else 64.
static void build_items_fp64(const LabelClasses& lc, const WorkList& wl) {
  std::vector<std::pair<int64_t, int32_t>> order; // (K steps of a tile, group)
  order.reserve(wl.groups.size());
  int64_t nitems = 0;
  for(size_t gi = 0; gi < wl.groups.size(); gi++) {
    const DevGroup& g = wl.groups[gi];
    if(g.task_begin == g.task_end) continue;
    int64_t work = 0;
    for(int t = g.task_begin; t < g.task_end; t++) {
      const DevTask& tk = wl.tasks[t];
      int64_t        k  = 1;
      for(int j = 0; j < lc.nk; j++) k *= tk.adims[lc.k_a[j]];
      for(int j = 0; j < lc.nar; j++) k *= tk.adims[lc.ar_a[j]];
      for(int j = 0; j < lc.nbr; j++) k *= tk.bdims[lc.br_b[j]];
      work += (k + BK - 1) / BK;
    }
    order.emplace_back(work, (int32_t) gi);
  }
  std::stable_sort(order.begin(), order.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  auto extents = [&](const DevGroup& g, int64_t& nbatch, int64_t& M, int64_t& N) {
    nbatch = M = N = 1;
    for(int j = 0; j < lc.nbatch; j++) nbatch *= g.cdims[lc.batch_c[j]];
    for(int j = 0; j < lc.nm; j++) M *= g.cdims[lc.m_c[j]];
    for(int j = 0; j < lc.nn; j++) N *= g.cdims[lc.n_c[j]];
  };
  double padded64 = 0, padded80 = 0; // MMA work of each width, tile padding included
  for(const auto& o: order) {
    int64_t nbatch, M, N;
    extents(wl.groups[o.second], nbatch, M, N);
    const double w = (double) o.first * nbatch * ((M + BM - 1) / BM);
    padded64 += w * ((N + 63) / 64) * 64;
    padded80 += w * ((N + 79) / 80) * 80;
  }
  const int BN = padded80 < padded64 ? 80 : 64;
  for(const auto& o: order) {
    int64_t nbatch, M, N;
    extents(wl.groups[o.second], nbatch, M, N);
    nitems += nbatch * ((M + BM - 1) / BM) * ((N + BN - 1) / BN);
  }
  TB_EXPECTS(nitems < (1ll << 31), "work list too large");
  wl.items_fp64.clear();
  wl.items_fp64.reserve((size_t) nitems);
  for(const auto& o: order) {
    int64_t nbatch, M, N;
    extents(wl.groups[o.second], nbatch, M, N);
    for(int64_t b = 0; b < nbatch; b++)
      for(int64_t m0 = 0; m0 < M; m0 += BM)
        for(int64_t n0 = 0; n0 < N; n0 += BN)
          wl.items_fp64.push_back(DevItem{o.second, (int32_t) b, (int32_t) m0, (int32_t) n0});
  }
  if(!wl.items_fp64.empty()) {
    TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&wl.d_items), sizeof(DevItem) * wl.items_fp64.size()));
    TB_CUDA(cudaMemcpy(wl.d_items, wl.items_fp64.data(), sizeof(DevItem) * wl.items_fp64.size(),
                       cudaMemcpyHostToDevice));
  }
  wl.items_bn    = BN;
  wl.items_built = true;
}

} // namespace tb
