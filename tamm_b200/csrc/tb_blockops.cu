// HBM-bound block kernels: permuted assign/accumulate (kernels::assign), fill (SetOp),
// axpby (flat AddOp / the bufacc axpy), deterministic dot / norm reductions, and the
// seeded counter-based generator.
#include "tb_internal.hpp"

#include <algorithm>
#include <cmath>

namespace tb {
namespace {

constexpr int kThreads = 256;

int grid_for(int64_t n, int per_thread) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int64_t want = (n + (int64_t) kThreads * per_thread - 1) / ((int64_t) kThreads * per_thread);
  int64_t cap  = (int64_t) sms * 8; // 8 resident CTAs of 256 threads per SM
  return (int) std::max<int64_t>(1, std::min<int64_t>(want, cap));
}

// ---- permuted assign: dst[sum i_k dld_k] (=|+=) scale * src[sum i_k sld_k] ----
// The destination is walked in its own row-major order so stores coalesce; the
// source side is gathered.  Index space up to 4-D as the reference's ip0..ip4.
struct AssignArgs {
  int     nd;
  int64_t dims[4], dld[4], sld[4];
  int64_t total;
};

__global__ void __launch_bounds__(kThreads) k_assign(AssignArgs a, double* __restrict__ dst,
                                                     double scale, const double* __restrict__ src,
                                                     int is_assign) {
  const int64_t stride = (int64_t) gridDim.x * blockDim.x;
  for(int64_t lin = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; lin < a.total; lin += stride) {
    int64_t x = lin, so = 0, doff = 0;
#pragma unroll
    for(int k = 3; k >= 0; k--) {
      if(k >= a.nd) continue;
      const int64_t d = a.dims[k];
      const int64_t q = x / d;
      const int64_t i = x - q * d;
      so += i * a.sld[k];
      doff += i * a.dld[k];
      x = q;
    }
    const double v = scale * __ldg(src + so);
    dst[doff]      = is_assign ? v : dst[doff] + v;
  }
}

// ---- pure permutation of >=2 modes whose last dst mode is not the last src mode:
// 32x32 tiles through shared memory so both the read and the write are coalesced.
struct TransArgs {
  int     nd;
  int64_t dims[4];      // dst-order loop dims
  int64_t dld[4], sld[4];
  int     p;            // loop position of the src stride-1 mode
  int64_t outer_total;  // product of dims except positions nd-1 and p
};

__global__ void __launch_bounds__(kThreads) k_assign_tiled(TransArgs a, double* __restrict__ dst,
                                                           double scale,
                                                           const double* __restrict__ src,
                                                           int is_assign) {
  __shared__ double tile[32][33];
  const int     q      = a.nd - 1;
  const int64_t Dq     = a.dims[q], Dp = a.dims[a.p];
  const int64_t tq     = (Dq + 31) / 32, tp = (Dp + 31) / 32;
  const int64_t ntiles = a.outer_total * tq * tp;
  for(int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int64_t x  = t;
    int64_t bq = x % tq;
    x /= tq;
    int64_t bp = x % tp;
    x /= tp;
    // outer index over modes other than p and q
    int64_t so = 0, doff = 0;
    for(int k = a.nd - 1; k >= 0; k--) {
      if(k == q || k == a.p) continue;
      const int64_t d = a.dims[k];
      const int64_t i = x % d;
      x /= d;
      so += i * a.sld[k];
      doff += i * a.dld[k];
    }
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5; // 32 x 8
    // read: consecutive threads along p (src stride 1)
    for(int r = ty; r < 32; r += 8) {
      const int64_t iq = bq * 32 + r, ip = bp * 32 + tx;
      if(iq < Dq && ip < Dp) tile[r][tx] = __ldg(src + so + iq * a.sld[q] + ip * a.sld[a.p]);
    }
    __syncthreads();
    // write: consecutive threads along q (dst stride 1)
    for(int r = ty; r < 32; r += 8) {
      const int64_t ip = bp * 32 + r, iq = bq * 32 + tx;
      if(iq < Dq && ip < Dp) {
        double*      dp = dst + doff + iq * a.dld[q] + ip * a.dld[a.p];
        const double v  = scale * tile[tx][r];
        *dp             = is_assign ? v : *dp + v;
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kThreads) k_fill(double* __restrict__ x, int64_t n, double v,
                                                   int is_assign) {
  const int64_t stride = (int64_t) gridDim.x * blockDim.x * 2;
  for(int64_t i = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) * 2; i < n; i += stride) {
    if(i + 1 < n && ((reinterpret_cast<uintptr_t>(x + i) & 15) == 0)) {
      double2 d;
      if(is_assign) d = make_double2(v, v);
      else {
        d = *reinterpret_cast<double2*>(x + i);
        d.x += v;
        d.y += v;
      }
      *reinterpret_cast<double2*>(x + i) = d;
    }
    else {
      for(int64_t j = i; j < i + 2 && j < n; j++) x[j] = is_assign ? v : x[j] + v;
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_axpby(double alpha, const double* __restrict__ x,
                                                    double beta, double* __restrict__ y, int64_t n) {
  const int64_t stride = (int64_t) gridDim.x * blockDim.x;
  for(int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    y[i] = beta == 0.0 ? alpha * x[i] : alpha * x[i] + beta * y[i];
}

// Deterministic dot: fixed grid, per-block partials in a fixed order, then one block
// folds the partials.  y == nullptr means x.x.
constexpr int kRedBlocks = 1024;

__global__ void __launch_bounds__(kThreads) k_dot_partial(const double* __restrict__ x,
                                                          const double* __restrict__ y, int64_t n,
                                                          double* __restrict__ part) {
  double        s      = 0.0;
  const int64_t stride = (int64_t) gridDim.x * blockDim.x;
  for(int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double a = x[i];
    s += a * (y ? y[i] : a);
  }
#pragma unroll
  for(int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double ws[kThreads / 32];
  if((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if(threadIdx.x == 0) {
    double t = 0.0;
    for(int w = 0; w < kThreads / 32; w++) t += ws[w];
    part[blockIdx.x] = t;
  }
}

__global__ void k_dot_final(const double* __restrict__ part, int np, double* __restrict__ out, double scale = 1.0,
                            int root = 0) {
  __shared__ double ws[32];
  double            s = 0.0;
  for(int i = threadIdx.x; i < np; i += blockDim.x) s += part[i];
#pragma unroll
  for(int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if(threadIdx.x == 0) {
    double t = 0.0;
    for(int w = 0; w < (int) (blockDim.x / 32); w++) t += ws[w];
    *out = scale * (root ? sqrt(t) : t);
  }
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ double u01(uint64_t seed_mix, uint64_t i) {
  const uint64_t h = splitmix64(seed_mix ^ (i * 0xD1B54A32D192ED03ull));
  return (double) (h >> 11) * (1.0 / 9007199254740992.0);
}

__global__ void __launch_bounds__(kThreads) k_fill_random(double* __restrict__ x, int64_t n,
                                                          uint64_t seed_mix, uint64_t first,
                                                          int dist, double p0, double p1) {
  const int64_t stride = (int64_t) gridDim.x * blockDim.x;
  for(int64_t q = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    const uint64_t i = first + (uint64_t) q;
    if(dist == 0) x[q] = p0 + (p1 - p0) * u01(seed_mix, i);
    else {
      double u1 = u01(seed_mix, 2 * i), u2 = u01(seed_mix, 2 * i + 1);
      if(u1 < 1e-300) u1 = 1e-300;
      x[q] = p0 + p1 * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    }
  }
}

uint64_t host_splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

} // namespace

AssignLoop plan_assign(const int64_t* ddims, const int* dlabels, int nd, const int64_t* sdims,
                       const int* slabels, int ns) {
  // kernels::assign (assign.hpp:467-485): permutation -> HPTT semantics, otherwise
  // ip_gen_loop (assign.hpp:312-373).  Both reduce to an nd-deep loop with dst and
  // src strides per loop label.
  TB_EXPECTS(nd >= 0 && nd <= kMaxModes && ns >= 0 && ns <= kMaxModes, "rank out of range");
  auto find = [](const int* v, int n, int x) {
    for(int i = 0; i < n; i++)
      if(v[i] == x) return i;
    return -1;
  };
  // are_permutations (perm.hpp:36-47)
  bool perm = (nd == ns);
  if(perm) {
    bool taken[kMaxModes] = {false};
    for(int i = 0; i < ns && perm; i++) {
      int p = find(dlabels, nd, slabels[i]);
      if(p < 0 || taken[p]) perm = false;
      else taken[p] = true;
    }
  }
  int64_t sld[kMaxModes + 1], dld[kMaxModes + 1];
  sld[ns] = 1;
  for(int i = ns - 1; i >= 0; i--) sld[i] = sld[i + 1] * sdims[i];
  dld[nd] = 1;
  for(int i = nd - 1; i >= 0; i--) dld[i] = dld[i + 1] * ddims[i];
  AssignLoop lp;
  lp.nd = nd;
  if(perm) {
    for(int i = 0; i < nd; i++) {
      int p = find(slabels, ns, dlabels[i]);
      TB_EXPECTS(ddims[i] == sdims[p], "dst dims are not a permutation of src dims");
    }
  }
  TB_EXPECTS(nd <= 4, "assign supports at most 4 destination modes (NOT_IMPLEMENTED beyond)");
  int loop_labels[2 * kMaxModes], nl = 0;
  for(int i = 0; i < nd; i++)
    if(find(loop_labels, nl, dlabels[i]) < 0) loop_labels[nl++] = dlabels[i];
  for(int i = 0; i < ns; i++)
    if(find(loop_labels, nl, slabels[i]) < 0) loop_labels[nl++] = slabels[i];
  TB_EXPECTS(nl >= nd, "repeated destination labels");
  for(int k = 0; k < nd; k++) {
    lp.dims[k] = 0;
    lp.sld[k]  = 0;
    lp.dld[k]  = 0;
    int ps     = find(slabels, ns, loop_labels[k]);
    if(ps >= 0) {
      lp.sld[k]  = sld[ps + 1];
      lp.dims[k] = sdims[ps];
    }
    int pd = find(dlabels, nd, loop_labels[k]);
    if(pd >= 0) {
      lp.dld[k]  = dld[pd + 1];
      lp.dims[k] = ddims[pd];
    }
  }
  return lp;
}

void launch_assign(const AssignLoop& lp, double* dst, double scale, const double* src,
                   int is_assign, cudaStream_t stream) {
  int64_t total = 1;
  for(int k = 0; k < lp.nd; k++) total *= lp.dims[k];
  if(total == 0) return;
  // A transposing permutation (dst's last loop mode is not src's stride-1 mode) goes
  // through the shared-memory tile kernel; everything else streams directly.
  int p = -1;
  for(int k = 0; k < lp.nd; k++)
    if(lp.sld[k] == 1 && lp.dims[k] > 1) p = k;
  const int q = lp.nd - 1;
  if(lp.nd >= 2 && p >= 0 && p != q && lp.dld[q] == 1 && lp.dims[q] >= 8 && lp.dims[p] >= 8) {
    TransArgs a;
    a.nd          = lp.nd;
    a.p           = p;
    a.outer_total = 1;
    for(int k = 0; k < 4; k++) {
      a.dims[k] = k < lp.nd ? lp.dims[k] : 1;
      a.dld[k]  = k < lp.nd ? lp.dld[k] : 0;
      a.sld[k]  = k < lp.nd ? lp.sld[k] : 0;
      if(k < lp.nd && k != p && k != q) a.outer_total *= lp.dims[k];
    }
    const int64_t ntiles = a.outer_total * ((lp.dims[q] + 31) / 32) * ((lp.dims[p] + 31) / 32);
    const int     grid   = (int) std::min<int64_t>(ntiles, 148 * 8);
    k_assign_tiled<<<grid, kThreads, 0, stream>>>(a, dst, scale, src, is_assign);
  }
  else {
    AssignArgs a;
    a.nd    = lp.nd;
    a.total = total;
    for(int k = 0; k < 4; k++) {
      a.dims[k] = k < lp.nd ? lp.dims[k] : 1;
      a.dld[k]  = k < lp.nd ? lp.dld[k] : 0;
      a.sld[k]  = k < lp.nd ? lp.sld[k] : 0;
    }
    k_assign<<<grid_for(total, 4), kThreads, 0, stream>>>(a, dst, scale, src, is_assign);
  }
  TB_CUDA(cudaGetLastError());
}

// min(want, the CTAs of `kernel` (kThreads threads, static shared memory) resident on
// the current device at once): one wave, each CTA taking an equal share.
template <class K>
int resident_grid(K kernel, int64_t want) {
  static int per_sm[64] = {0};
  int        dev        = 0;
  TB_CUDA(cudaGetDevice(&dev));
  int& k = per_sm[dev < 64 ? dev : 63];
  if(k == 0) {
    int r = 0;
    TB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, kernel, kThreads, 0));
    k = std::max(r, 1);
  }
  int nsm = 0;
  TB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  return (int) std::max<int64_t>(1, std::min<int64_t>(want, (int64_t) nsm * k));
}

constexpr int kAsgElems  = 8;                           // elements per thread and work unit
constexpr int kAsgN      = kThreads * kAsgElems;        // elements per work unit at most
constexpr int kAsgQ      = 64;                          // sub-tile extent along q at most
constexpr int kAsgP      = 32;                          // sub-tile extent along p at most
constexpr int kAsgStage  = kAsgQ * (kAsgP + 1);         // doubles of one shared-memory stage
constexpr int kAsgMaxSub = 32;                          // sub-tiles per work unit at most
constexpr int kAsgRows   = 256;                         // streamed rows per work unit at most

// Multiplier of x / d for 0 <= x < 2^32 and 2 <= d < 2^32: umul64hi(x, ceil(2^64 / d))
// (Granlund and Montgomery, division by invariant integers using multiplication: the
// rounding error x * (m - 2^64 / d) / 2^64 < 2^-32 stays below 1 / d).  0 for d = 1.
static uint64_t asg_magic64(int64_t d) { return d <= 1 ? 0 : ~uint64_t(0) / (uint64_t) d + 1; }

BlockAssign make_block_assign(const AssignLoop& lp, int64_t dst_off, int64_t src_off, int64_t first) {
  BlockAssign b{};
  b.dst_off    = dst_off;
  b.src_off    = src_off;
  b.nd         = lp.nd;
  b.first      = first;
  int64_t total = 1;
  for(int k = 0; k < lp.nd; k++) total *= lp.dims[k];
  int p = -1;
  for(int k = 0; k < lp.nd; k++)
    if(lp.sld[k] == 1 && lp.dims[k] > 1) p = k;
  const int q = lp.nd - 1;
  const bool tiled = lp.nd >= 2 && p >= 0 && p != q && lp.dld[q] == 1 && lp.dims[q] >= 8 && lp.dims[p] >= 8;
  b.p   = tiled ? p : -1;
  b.upr = 1;
  b.nbq = b.nbp = 1;
  b.per_unit    = 1;
  b.tq = b.tp   = 1;
  int64_t units = 0;
  if(total > 0) {
    // counts, strides and offsets within one block pair are 32-bit
    int64_t ssize = 1, dsize = 1;
    for(int k = 0; k < lp.nd; k++) {
      ssize += (lp.dims[k] - 1) * lp.sld[k];
      dsize += (lp.dims[k] - 1) * lp.dld[k];
    }
    TB_EXPECTS(ssize < (int64_t(1) << 31) && dsize < (int64_t(1) << 31) && total < (int64_t(1) << 31),
               "block too large");
    for(int k = 0; k < 4; k++) {
      b.dims[k] = (int32_t) (k < lp.nd ? lp.dims[k] : 1);
      b.dld[k]  = (int32_t) (k < lp.nd ? lp.dld[k] : 0);
      b.sld[k]  = (int32_t) (k < lp.nd ? lp.sld[k] : 0);
      b.mag[k]  = asg_magic64(b.dims[k]);
    }
    if(tiled) { // sub-tiles of nearly equal extents: a ragged block costs few idle lanes
      int64_t outer = 1;
      for(int k = 0; k < lp.nd; k++)
        if(k != p && k != q) outer *= lp.dims[k];
      const int64_t nbq = (lp.dims[q] + kAsgQ - 1) / kAsgQ, nbp = (lp.dims[p] + kAsgP - 1) / kAsgP;
      const int64_t tq = (lp.dims[q] + nbq - 1) / nbq, tp = (lp.dims[p] + nbp - 1) / nbp;
      b.nbq      = (int32_t) nbq;
      b.nbp      = (int32_t) nbp;
      b.tq       = (int32_t) tq;
      b.tp       = (int32_t) tp;
      b.nsub     = (int32_t) (outer * nbq * nbp);
      b.per_unit = (int32_t) std::max<int64_t>(
          1, std::min<int64_t>({(int64_t) kAsgMaxSub, kAsgN / (tq * tp), kAsgStage / (tq * (tp | 1))}));
      units = (b.nsub + b.per_unit - 1) / b.per_unit;
    }
    else { // rows of the destination's last mode (one row of length 1 for a scalar block)
      const int64_t len = lp.nd > 0 ? lp.dims[q] : 1;
      b.tq              = (int32_t) len;
      b.nsub            = (int32_t) (total / len);
      if(len <= kAsgN) {
        b.per_unit = (int32_t) std::min<int64_t>(kAsgRows, kAsgN / len);
        units      = (b.nsub + b.per_unit - 1) / b.per_unit;
      }
      else {
        b.upr = (int32_t) ((len + kAsgN - 1) / kAsgN);
        units = (int64_t) b.nsub * b.upr;
      }
    }
    b.mag[4] = asg_magic64(b.nbq);
    b.mag[5] = asg_magic64(b.nbp);
  }
  TB_EXPECTS(units < (int64_t(1) << 31), "block pair too large");
  b.units = (int32_t) units;
  return b;
}

namespace {

// x / d for 0 <= x < 2^11 and 1 <= d <= 2^20, with m = asg_magic(d): umulhi(x, ceil(2^32 / d))
// (Granlund and Montgomery; the rounding error x * (m - 2^32 / d) / 2^32 < 2^-21 stays
// below 1 / d).  d = 1 has no 32-bit multiplier and returns x.
__device__ __forceinline__ unsigned asg_magic(unsigned d) { return d == 1 ? 0u : 0xFFFFFFFFu / d + 1; }
__device__ __forceinline__ int asg_div(int x, unsigned m) { return m == 0 ? x : (int) __umulhi((unsigned) x, m); }
// x / d for 0 <= x < 2^31 with the host's 64-bit multiplier (asg_magic64)
__device__ __forceinline__ int asg_div64(int x, uint64_t m) {
  return m == 0 ? x : (int) __umul64hi((uint64_t) (uint32_t) x, m);
}

__device__ __forceinline__ void asg_cp8(uint32_t saddr, const double* g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void asg_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void asg_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Per-unit records, kept in one slot of a three-slot ring: origins (source and
// destination offsets within the pair's blocks) and extents (nq | np << 16) of a
// transposed unit's sub-tiles, or the row origins of a streamed unit.
struct AsgRing {
  int so[3][kAsgRows];
  int dof[3][kAsgRows];
  int ext[3][kAsgMaxSub];
};

// Elements of unit lu of pair a: sub-tiles x tq x tp, rows x row length, or one chunk of a long row.
__device__ __forceinline__ int asg_unit_elems(const BlockAssign& a, int lu) {
  if(a.p >= 0) return min(a.per_unit, a.nsub - lu * a.per_unit) * a.tq * a.tp;
  if(a.upr == 1) return min(a.per_unit, a.nsub - lu * a.per_unit) * a.tq;
  const int c = lu % a.upr;
  return min(kAsgN, a.tq - c * kAsgN);
}

// Records of unit lu of pair a into ring slot s (threads below the unit's record count).
__device__ __forceinline__ void asg_records(const BlockAssign& a, int lu, AsgRing& r, int s) {
  const int t = threadIdx.x;
  if(a.p >= 0) {
    const int q = a.nd - 1, p = a.p, t0 = lu * a.per_unit;
    if(t < a.per_unit && t0 + t < a.nsub) {
      int       x  = t0 + t;
      int       y  = asg_div64(x, a.mag[4]);
      const int bq = x - y * a.nbq;
      x            = asg_div64(y, a.mag[5]);
      const int bp = y - x * a.nbp;
      int       so = 0, doff = 0;
      for(int k = a.nd - 1; k >= 0; k--) {
        if(k == q || k == p) continue;
        const int z = asg_div64(x, a.mag[k]), i = x - z * a.dims[k];
        x           = z;
        so += i * a.sld[k];
        doff += i * a.dld[k];
      }
      const int q0 = bq * a.tq, p0 = bp * a.tp;
      r.so[s][t]   = so + q0 * a.sld[q] + p0;
      r.dof[s][t]  = doff + q0 + p0 * a.dld[p];
      r.ext[s][t]  = min(a.tq, a.dims[q] - q0) | (min(a.tp, a.dims[p] - p0) << 16);
    }
    return;
  }
  const int r0 = a.upr == 1 ? lu * a.per_unit : lu / a.upr;
  const int nr = a.upr == 1 ? min(a.per_unit, a.nsub - r0) : 1;
  if(t < nr) {
    int x = r0 + t, so = 0, doff = 0;
    for(int k = a.nd - 2; k >= 0; k--) {
      const int z = asg_div64(x, a.mag[k]), i = x - z * a.dims[k];
      x           = z;
      so += i * a.sld[k];
      doff += i * a.dld[k];
    }
    r.so[s][t]  = so;
    r.dof[s][t] = doff;
  }
}

// Issue the source loads of unit lu of pair a into a shared-memory stage (8-byte
// cp.async per element, this thread's elements only): a transposed unit's sub-tiles
// row by row along p (odd row pitch), a streamed unit in element order.
__device__ __forceinline__ void asg_load(const BlockAssign& a, int lu, const AsgRing& r, int s,
                                         const double* __restrict__ src, uint32_t stage) {
  const double* s0 = src + a.src_off;
  const int     n  = asg_unit_elems(a, lu);
  if(a.p >= 0) {
    const int      TQ = a.tq, TP = a.tp, pitch = TP | 1, sq = a.sld[a.nd - 1];
    const unsigned mq = asg_magic(TQ), mp = asg_magic(TP);
#pragma unroll
    for(int j = 0; j < kAsgElems; j++) {
      const int e = threadIdx.x + j * kThreads;
      if(e < n) {
        const int row = asg_div(e, mp), ip = e - row * TP;
        const int k = asg_div(row, mq), iq = row - k * TQ;
        const int ext = r.ext[s][k];
        if(iq < (ext & 0xFFFF) && ip < (ext >> 16))
          asg_cp8(stage + (uint32_t) (row * pitch + ip) * 8u, s0 + r.so[s][k] + iq * sq + ip);
      }
    }
    return;
  }
  const int      L  = a.tq;
  const int      sq = a.nd > 0 ? a.sld[a.nd - 1] : 0;
  const unsigned mL = asg_magic(L);
  const int      c0 = a.upr == 1 ? 0 : (lu % a.upr) * kAsgN;
#pragma unroll
  for(int j = 0; j < kAsgElems; j++) {
    const int e = threadIdx.x + j * kThreads;
    if(e < n) {
      const int row = a.upr == 1 ? asg_div(e, mL) : 0, col = c0 + e - row * L;
      asg_cp8(stage + (uint32_t) e * 8u, s0 + r.so[s][row] + col * sq);
    }
  }
}

} // namespace

// The block pairs of an AddOp in one launch.  Work units (a batch of sub-tiles of one
// pair's transposed (q, p) plane, or rows of a streamed pair) are split into equal
// contiguous ranges, one per CTA.  Each CTA runs its units through a two-stage
// pipeline: while unit u is written, unit u+1's source elements are already on their
// way into the other shared-memory stage (cp.async) and unit u+2's records are
// computed; unit u's old destination values are loaded before the wait for its
// source, so both reads of a unit overlap.  A transposing unit lands its sub-tiles
// along the source's stride-1 mode p (odd row pitch) and is written row by row along
// the destination's stride-1 mode q; a streamed unit is written in element order.
// Sub-tiles have the blocks' own extents (at most 64 x 32, nearly equal), so few
// lanes go to padding.  All index arithmetic is 32-bit, divisions by the blocks'
// extents multiply by constants the host computed.
__global__ void __launch_bounds__(kThreads, 4) k_assign_blocks(double* __restrict__ dst, double scale,
                                                               const double* __restrict__ src,
                                                               const BlockAssign* __restrict__ blocks, int nblocks,
                                                               int nunits, int is_assign) {
  __shared__ __align__(16) double tile[2][kAsgStage];
  __shared__ AsgRing              ring;
  __shared__ int                  s_pair;
  const int u0 = (int) ((int64_t) nunits * blockIdx.x / gridDim.x);
  const int u1 = (int) ((int64_t) nunits * (blockIdx.x + 1) / gridDim.x);
  if(u0 >= u1) return;
  if(threadIdx.x == 0) { // the pair holding unit u0: last pair with first <= u0
    int lo = 0, hi = nblocks - 1;
    while(lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if(blocks[mid].first <= u0) lo = mid;
      else hi = mid - 1;
    }
    s_pair = lo;
  }
  __syncthreads();
  const uint32_t st0 = (uint32_t) __cvta_generic_to_shared(&tile[0][0]);
  const uint32_t st1 = (uint32_t) __cvta_generic_to_shared(&tile[1][0]);
  auto pair_of = [&](int pi, int u) {
    while(u >= blocks[pi].first + blocks[pi].units) pi++;
    return pi;
  };
  int pi = pair_of(s_pair, u0);
  asg_records(blocks[pi], u0 - (int) blocks[pi].first, ring, 0);
  __syncthreads();
  asg_load(blocks[pi], u0 - (int) blocks[pi].first, ring, 0, src, st0);
  asg_commit();
  int pn = pi; // pair of unit u + 1
  if(u0 + 1 < u1) {
    pn = pair_of(pi, u0 + 1);
    asg_records(blocks[pn], u0 + 1 - (int) blocks[pn].first, ring, 1);
  }
  __syncthreads();
  int slot = 0, stage = 0;
  for(int u = u0; u < u1; u++) {
    const int sn = slot == 2 ? 0 : slot + 1, sn2 = sn == 2 ? 0 : sn + 1;
    if(u + 1 < u1) asg_load(blocks[pn], u + 1 - (int) blocks[pn].first, ring, sn, src, stage ? st0 : st1);
    asg_commit();
    const int pn2 = u + 2 < u1 ? pair_of(pn, u + 2) : pn;
    if(u + 2 < u1) asg_records(blocks[pn2], u + 2 - (int) blocks[pn2].first, ring, sn2);
    const BlockAssign& a  = blocks[pi];
    const int          lu = u - (int) a.first;
    const int          n  = asg_unit_elems(a, lu);
    double* const      d0 = dst + a.dst_off;
    double             old[kAsgElems];
    int                out[kAsgElems], at[kAsgElems]; // destination offset (-1: none), stage slot
    if(a.p >= 0) {
      const int      TQ = a.tq, TP = a.tp, pitch = TP | 1, dp = a.dld[a.p];
      const unsigned mq = asg_magic(TQ), mp = asg_magic(TP);
#pragma unroll
      for(int j = 0; j < kAsgElems; j++) {
        const int e = threadIdx.x + j * kThreads;
        out[j]      = -1;
        at[j]       = 0;
        if(e < n) {
          const int row = asg_div(e, mq), iq = e - row * TQ;
          const int k = asg_div(row, mp), ip = row - k * TP;
          const int ext = ring.ext[slot][k];
          if(iq < (ext & 0xFFFF) && ip < (ext >> 16)) {
            out[j] = ring.dof[slot][k] + ip * dp + iq;
            at[j]  = (k * TQ + iq) * pitch + ip;
          }
        }
      }
    }
    else {
      const int      L  = a.tq;
      const int      dq = a.nd > 0 ? a.dld[a.nd - 1] : 0;
      const unsigned mL = asg_magic(L);
      const int      c0 = a.upr == 1 ? 0 : (lu % a.upr) * kAsgN;
#pragma unroll
      for(int j = 0; j < kAsgElems; j++) {
        const int e = threadIdx.x + j * kThreads;
        out[j]      = -1;
        at[j]       = e;
        if(e < n) {
          const int row = a.upr == 1 ? asg_div(e, mL) : 0, col = c0 + e - row * L;
          out[j]        = ring.dof[slot][row] + col * dq;
        }
      }
    }
#pragma unroll
    for(int j = 0; j < kAsgElems; j++) old[j] = (!is_assign && out[j] >= 0) ? d0[out[j]] : 0.0;
    asg_wait_prev(); // this thread's copies of unit u have landed
    __syncthreads(); // and every other thread's
    const double* t = tile[stage];
#pragma unroll
    for(int j = 0; j < kAsgElems; j++) // product rounded before the add, as in a plain loop
      if(out[j] >= 0) {
        const double v = __dmul_rn(scale, t[at[j]]);
        d0[out[j]]     = is_assign ? v : old[j] + v;
      }
    __syncthreads(); // stage and slot free for units u + 2 and u + 3
    pi    = pn;
    pn    = pn2;
    slot  = sn;
    stage ^= 1;
  }
}

void launch_assign_blocks(double* dst, double scale, const double* src, const BlockAssign* blocks, int nblocks,
                          int64_t nunits, int is_assign, cudaStream_t stream) {
  if(nblocks <= 0 || nunits <= 0) return;
  TB_EXPECTS(nunits < (int64_t(1) << 31), "too many work units in one add");
  k_assign_blocks<<<resident_grid(k_assign_blocks, nunits), kThreads, 0, stream>>>(dst, scale, src, blocks, nblocks,
                                                                                     (int) nunits, is_assign);
  TB_CUDA(cudaGetLastError());
}

void launch_fill(double* x, int64_t n, double value, int is_assign, cudaStream_t stream) {
  if(n <= 0) return;
  k_fill<<<grid_for(n, 8), kThreads, 0, stream>>>(x, n, value, is_assign);
  TB_CUDA(cudaGetLastError());
}

constexpr int kSegVec = 4; // 16-byte accesses in flight per thread

// A CTA's share of a segment list: elements [N b / G, N (b + 1) / G) of the runs'
// concatenation (N elements in all, G CTAs), walked run by run; body(dst offset, src
// offset, lo, hi) gets the part [lo, hi) of each run it overlaps.
template <class Body>
__device__ __forceinline__ void walk_segments(const int64_t* __restrict__ seg, int nseg, Body body) {
  __shared__ int s_first;
  const int64_t  N  = seg[4 * (nseg - 1) + 3] + seg[4 * (nseg - 1) + 2];
  const int64_t  e0 = N * blockIdx.x / gridDim.x, e1 = N * (blockIdx.x + 1) / gridDim.x;
  if(e0 >= e1) return;
  if(threadIdx.x == 0) { // last run with first <= e0
    int lo = 0, hi = nseg - 1;
    while(lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if(seg[4 * mid + 3] <= e0) lo = mid;
      else hi = mid - 1;
    }
    s_first = lo;
  }
  __syncthreads();
  for(int r = s_first; r < nseg && seg[4 * r + 3] < e1; r++) {
    const int64_t f = seg[4 * r + 3], n = seg[4 * r + 2];
    const int64_t lo = max(e0, f) - f, hi = min(e1, f + n) - f;
    if(lo < hi) body(seg[4 * r], seg[4 * r + 1], lo, hi);
  }
}

// y[lo, hi) = g(x[lo, hi), y[lo, hi)) elementwise (x may be null: zeros; x may equal
// y; y read only when READY): one element before the first 16-byte boundary of y, then
// double2 accesses with kSegVec in flight per thread when x shares y's alignment, else
// scalar ones.
template <bool READY, class G>
__device__ __forceinline__ void seg_apply(double* y, const double* x, int64_t lo, int64_t hi, G g) {
  int64_t a = lo;
  if((reinterpret_cast<uintptr_t>(y + a) & 15) != 0) {
    if(threadIdx.x == 0) y[a] = g(x ? x[a] : 0.0, READY ? y[a] : 0.0);
    a++;
  }
  if(a >= hi) return;
  if(x == nullptr || (reinterpret_cast<uintptr_t>(x + a) & 15) == 0) {
    const int64_t  nv = (hi - a) >> 1;
    double2* const y2 = reinterpret_cast<double2*>(y + a);
    const double2* x2 = x ? reinterpret_cast<const double2*>(x + a) : nullptr;
    for(int64_t i = threadIdx.x; i < nv; i += (int64_t) kThreads * kSegVec) {
      double2 xv[kSegVec], yv[kSegVec];
#pragma unroll
      for(int j = 0; j < kSegVec; j++) {
        const int64_t k = i + (int64_t) j * kThreads;
        xv[j] = yv[j] = make_double2(0.0, 0.0);
        if(k < nv) {
          if(x2) xv[j] = x2[k];
          if(READY) yv[j] = y2[k];
        }
      }
#pragma unroll
      for(int j = 0; j < kSegVec; j++) {
        const int64_t k = i + (int64_t) j * kThreads;
        if(k < nv) y2[k] = make_double2(g(xv[j].x, yv[j].x), g(xv[j].y, yv[j].y));
      }
    }
    if(threadIdx.x == 0 && a + 2 * nv < hi) y[hi - 1] = g(x ? x[hi - 1] : 0.0, READY ? y[hi - 1] : 0.0);
  }
  else {
    for(int64_t i = a + threadIdx.x; i < hi; i += (int64_t) kThreads * kSegVec) {
      double xv[kSegVec], yv[kSegVec];
#pragma unroll
      for(int j = 0; j < kSegVec; j++) {
        const int64_t k = i + (int64_t) j * kThreads;
        xv[j] = yv[j] = 0.0;
        if(k < hi) {
          xv[j] = x[k];
          if(READY) yv[j] = y[k];
        }
      }
#pragma unroll
      for(int j = 0; j < kSegVec; j++) {
        const int64_t k = i + (int64_t) j * kThreads;
        if(k < hi) y[k] = g(xv[j], yv[j]);
      }
    }
  }
}

std::vector<int64_t> seg_list(const std::vector<int64_t>& tri) {
  std::vector<int64_t> out;
  int64_t              first = 0;
  for(size_t i = 0; i + 2 < tri.size(); i += 3) {
    const int64_t d = tri[i], s = tri[i + 1], n = tri[i + 2];
    if(n <= 0) continue;
    const size_t m = out.size();
    if(m > 0 && out[m - 4] + out[m - 2] == d &&
       ((s < 0 && out[m - 3] < 0) || (s >= 0 && out[m - 3] >= 0 && out[m - 3] + out[m - 2] == s)))
      out[m - 2] += n;
    else {
      out.push_back(d);
      out.push_back(s);
      out.push_back(n);
      out.push_back(first);
    }
    first += n;
  }
  return out;
}

__global__ void __launch_bounds__(kThreads) k_fill_blocks(double* __restrict__ x, const int64_t* __restrict__ segs,
                                                          int nseg, double v, int is_assign) {
  walk_segments(segs, nseg, [&](int64_t off, int64_t, int64_t lo, int64_t hi) {
    if(is_assign) seg_apply<false>(x + off, nullptr, lo, hi, [v](double, double) { return v; });
    else seg_apply<true>(x + off, nullptr, lo, hi, [v](double, double y) { return y + v; });
  });
}

void launch_fill_blocks(double* x, const int64_t* segs, int nseg, int64_t total, double value, int is_assign,
                        cudaStream_t stream) {
  if(nseg <= 0 || total <= 0) return;
  k_fill_blocks<<<resident_grid(k_fill_blocks, (total + 4095) / 4096), kThreads, 0, stream>>>(x, segs, nseg, value,
                                                                                              is_assign);
  TB_CUDA(cudaGetLastError());
}

__device__ __forceinline__ double map_fn(int fn, double x, double p) {
  switch(fn) {
    case TB_MAP_COPY: return x;
    case TB_MAP_SCALE: return p * x;
    case TB_MAP_SET: return p;
    case TB_MAP_SQUARE: return x * x;
    case TB_MAP_SQRT: return sqrt(x);
    case TB_MAP_LOG: return log(x);
    case TB_MAP_LOG10: return log10(x);
    case TB_MAP_INVERSE: return 1.0 / x;
    case TB_MAP_POW: return pow(x, p);
    default: return fabs(x);
  }
}

// Element function over a segment list, each CTA on an equal share of its elements.
__global__ void __launch_bounds__(kThreads) k_map_blocks(double* __restrict__ dst, const double* __restrict__ src,
                                                         const int64_t* __restrict__ segs, int nseg, int fn,
                                                         double p) {
  walk_segments(segs, nseg, [&](int64_t doff, int64_t soff, int64_t lo, int64_t hi) {
    seg_apply<false>(dst + doff, soff >= 0 ? src + soff : nullptr, lo, hi,
              [fn, p](double x, double) { return map_fn(fn, x, p); });
  });
}

void launch_map_blocks(double* dst, const double* src, const int64_t* segs, int nseg, int64_t total, int fn,
                       double p, cudaStream_t stream) {
  if(nseg <= 0 || total <= 0) return;
  k_map_blocks<<<resident_grid(k_map_blocks, (total + 4095) / 4096), kThreads, 0, stream>>>(dst, src, segs, nseg, fn,
                                                                                             p);
  TB_CUDA(cudaGetLastError());
}

// One pass over the blocks of a read-only tensor: a CTA row (blockIdx.y) per block,
// 16-byte loads where aligned, one OR per CTA that saw a nonzero element.
__global__ void __launch_bounds__(kThreads) k_block_nonzero(const double* __restrict__ x,
                                                            const int64_t* __restrict__ pairs, int nblocks,
                                                            uint32_t* __restrict__ nonzero) {
  for(int blk = blockIdx.y; blk < nblocks; blk += gridDim.y) {
    const double* const xb     = x + pairs[2 * blk];
    const int64_t       n      = pairs[2 * blk + 1];
    const int64_t       stride = (int64_t) gridDim.x * blockDim.x * 2;
    int                 any    = 0;
    for(int64_t i = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) * 2; i < n && !any; i += stride) {
      if(i + 1 < n && ((reinterpret_cast<uintptr_t>(xb + i) & 15) == 0)) {
        const double2 d = __ldcs(reinterpret_cast<const double2*>(xb + i));
        any             = (d.x != 0.0) | (d.y != 0.0);
      }
      else
        for(int64_t j = i; j < i + 2 && j < n; j++) any |= (xb[j] != 0.0);
    }
    if(__syncthreads_or(any) && threadIdx.x == 0) atomicOr(nonzero + blk, 1u);
  }
}

void launch_block_nonzero(const double* x, const int64_t* pairs, int nblocks, uint32_t* nonzero,
                          cudaStream_t stream) {
  if(nblocks <= 0) return;
  TB_CUDA(cudaMemsetAsync(nonzero, 0, sizeof(uint32_t) * nblocks, stream));
  const dim3 grid(16, (unsigned) std::min(nblocks, 4096));
  k_block_nonzero<<<grid, kThreads, 0, stream>>>(x, pairs, nblocks, nonzero);
  TB_CUDA(cudaGetLastError());
}

void launch_axpby(double alpha, const double* x, double beta, double* y, int64_t n,
                  cudaStream_t stream) {
  if(n <= 0) return;
  k_axpby<<<grid_for(n, 4), kThreads, 0, stream>>>(alpha, x, beta, y, n);
  TB_CUDA(cudaGetLastError());
}

double reduce_dot(const double* x, const double* y, int64_t n, cudaStream_t stream) {
  if(n <= 0) return 0.0;
  double* part = nullptr;
  TB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&part), sizeof(double) * (kRedBlocks + 1), stream));
  k_dot_partial<<<kRedBlocks, kThreads, 0, stream>>>(x, y, n, part);
  k_dot_final<<<1, 1024, 0, stream>>>(part, kRedBlocks, part + kRedBlocks);
  double h = 0.0;
  TB_CUDA(cudaMemcpyAsync(&h, part + kRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, stream));
  TB_CUDA(cudaFreeAsync(part, stream));
  TB_CUDA(cudaStreamSynchronize(stream));
  return h;
}

// Orbital-energy denominators over the admitted blocks of a tensor: for element
// (x_0, ..., x_last) of a block, D = sum_m s_m * eps[first_m + x_m].  The work is
// cut into units of consecutive rows of one block (a row: all modes but the last;
// up to kDenRows rows, about kDenomUnitElems elements), and a persistent grid walks
// the units: the CTA forms the row part of D for each of the unit's rows in shared
// memory (the last mode's part is tabulated once per unit), then streams the unit's
// elements with coalesced loads, eight in flight per thread.  A last mode of at most
// kThreads columns gives each thread one fixed column (its part of D in a register)
// and floor(kThreads / columns) rows per pass; a longer one steps (row, column)
// through the unit without divisions.
//   ENERGY:  part[cta] = sum w^2 / D  (w = t; each CTA sums its units in a fixed
//            order, k_denom_energy_final sums the CTAs in a fixed order)
//   update:  t += scale * r / D
constexpr int kDenCols = 1024; // last-mode extents tabulated in shared memory
constexpr int kDenRows = kDenomUnitRows; // rows of one unit (row parts of D in shared memory)

template<bool ENERGY>
__global__ void __launch_bounds__(kThreads) k_denom(double* __restrict__ t, const double* __restrict__ r, double scale,
                                                    const DenomBlock* __restrict__ blocks,
                                                    const DenomUnit* __restrict__ units, int nunits, int nmodes,
                                                    const double* __restrict__ eps, DenomSigns sg,
                                                    double* __restrict__ part) {
  __shared__ double drow[kDenRows];
  __shared__ double dcol[kDenCols];
  __shared__ double s_sg[kMaxModes];
  constexpr int     U    = 8; // loads in flight per thread
  const int         tid  = threadIdx.x;
  const int         last = nmodes - 1;
  double            s    = 0.0;
  // the signs go to shared memory by static indices, and the blocks' fields are read
  // through a pointer: indexing a copy of either by a runtime mode would put it in
  // local memory (published by the first barrier of the unit loop)
#pragma unroll
  for(int m = 0; m < kMaxModes; m++)
    if(tid == m) s_sg[m] = sg.s[m];
  // one element: its value(s) and its denominator
  auto elem = [&](int64_t i, double v, double w, double D) {
    if constexpr(ENERGY) s += v * v * recip_nr(D);
    else t[i] = v + scale * w * recip_nr(D);
  };
  auto load = [&](int64_t i, double& v, double& w) {
    if constexpr(ENERGY) v = __ldg(t + i);
    else {
      v = t[i];
      w = __ldg(r + i);
    }
  };
  for(int ui = blockIdx.x; ui < nunits; ui += gridDim.x) {
    const DenomUnit                u  = units[ui];
    const DenomBlock* __restrict__ bp = blocks + u.block;
    const int32_t                  nc = (int32_t) bp->dims[last];
    const bool                     tab = nc <= kDenCols;
    const double*                  el  = eps + bp->first[last];
    __syncthreads(); // the previous unit is done with drow / dcol
    const double slst = s_sg[last];
    if(tab)
      for(int c = tid; c < nc; c += kThreads) dcol[c] = slst * __ldg(el + c);
    for(int i = tid; i < u.rows; i += kThreads) {
      int32_t x = (int32_t) (u.r0 + i); // a block holds fewer than 2^31 elements
      double  d = 0.0;
      for(int m = last - 1; m >= 0; m--) {
        const int32_t n = (int32_t) bp->dims[m], q = x / n;
        d += s_sg[m] * __ldg(eps + bp->first[m] + (x - q * n));
        x = q;
      }
      drow[i] = d;
    }
    __syncthreads();
    const int64_t base = bp->off + u.r0 * (int64_t) nc;
    if(nc <= kThreads) { // fixed column per thread, P rows per pass of A elements
      const int P = kThreads / nc, A = P * nc;
      if(tid < A) {
        const int     ro = tid / nc;
        const double  dc = dcol[tid - ro * nc];
        const int     nk = (u.rows - ro + P - 1) / P; // rows ro, ro + P, ... of the unit
        const int64_t e0 = base + tid;
        int           k  = 0;
        for(; k + U <= nk; k += U) {
          double v[U], w[U];
#pragma unroll
          for(int j = 0; j < U; j++) load(e0 + (int64_t) (k + j) * A, v[j], w[j]);
#pragma unroll
          for(int j = 0; j < U; j++) elem(e0 + (int64_t) (k + j) * A, v[j], w[j], drow[ro + (k + j) * P] + dc);
        }
        for(; k < nk; k++) {
          double v, w;
          load(e0 + (int64_t) k * A, v, w);
          elem(e0 + (int64_t) k * A, v, w, drow[ro + k * P] + dc);
        }
      }
    }
    else { // long rows: step (row, column) by kThreads elements, no divisions
      const int32_t nel = u.rows * nc;
      int32_t       rr = 0, cc = tid, e = tid;
      auto          den = [&]() {
        const double D = drow[rr] + (tab ? dcol[cc] : slst * __ldg(el + cc));
        cc += kThreads;
        if(cc >= nc) {
          cc -= nc;
          rr++;
        }
        return D;
      };
      for(; e + (U - 1) * kThreads < nel; e += U * kThreads) {
        double v[U], w[U];
#pragma unroll
        for(int j = 0; j < U; j++) load(base + e + j * kThreads, v[j], w[j]);
#pragma unroll
        for(int j = 0; j < U; j++) elem(base + e + j * kThreads, v[j], w[j], den());
      }
      for(; e < nel; e += kThreads) {
        double v, w;
        load(base + e, v, w);
        elem(base + e, v, w, den());
      }
    }
  }
  if constexpr(ENERGY) {
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double ws[kThreads / 32];
    if((tid & 31) == 0) ws[tid >> 5] = s;
    __syncthreads();
    if(tid == 0) {
      double v = 0.0;
      for(int i = 0; i < kThreads / 32; i++) v += ws[i];
      part[blockIdx.x] = v;
    }
  }
}

// Persistent grid of the denominator kernels: as many CTAs as fit on the GPU at once,
// at most one per unit.
template<bool ENERGY>
int denom_grid(int nunits) {
  static int per_sm[64] = {0};
  int        dev        = 0;
  TB_CUDA(cudaGetDevice(&dev));
  int& k = per_sm[dev < 64 ? dev : 63];
  if(k == 0) {
    TB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, k_denom<ENERGY>, kThreads, 0));
    k = std::max(k, 1);
  }
  int nsm = 0;
  TB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  return std::min(nunits, nsm * k);
}

__global__ void k_denom_energy_final(const double* __restrict__ part, int np, double scale, double* __restrict__ out) {
  __shared__ double ws[32];
  double            s = 0.0;
  for(int i = threadIdx.x; i < np; i += blockDim.x) s += part[i];
#pragma unroll
  for(int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if(threadIdx.x == 0) {
    double t = 0.0;
    for(int w = 0; w < (int) (blockDim.x / 32); w++) t += ws[w];
    *out += scale * t;
  }
}

__global__ void k_set_scalar(double* out, double v) { *out = v; }

void launch_denom_energy(const double* w, double scale, const DenomBlock* blocks, const DenomUnit* units,
                         int nunits, int nmodes, const double* eps, DenomSigns signs, double* part, double* out,
                         cudaStream_t stream) {
  const int grid = nunits > 0 ? denom_grid<true>(nunits) : 0;
  if(grid > 0)
    k_denom<true><<<grid, kThreads, 0, stream>>>(const_cast<double*>(w), nullptr, 0.0, blocks, units, nunits, nmodes,
                                                 eps, signs, part);
  k_denom_energy_final<<<1, 1024, 0, stream>>>(part, grid, scale, out);
  TB_CUDA(cudaGetLastError());
}

void launch_energy_final(const double* part, int64_t np, double scale, double* out, cudaStream_t stream) {
  if(np <= 0) return;
  TB_EXPECTS(np < (int64_t(1) << 31), "too many partial sums");
  k_denom_energy_final<<<1, 1024, 0, stream>>>(part, (int) np, scale, out);
  TB_CUDA(cudaGetLastError());
}

void launch_set_scalar(double* out, double v, cudaStream_t stream) {
  k_set_scalar<<<1, 1, 0, stream>>>(out, v);
  TB_CUDA(cudaGetLastError());
}

void launch_dot_to(const double* x, const double* y, int64_t n, double scale, int root, double* out, double* part,
                   cudaStream_t stream) {
  if(n <= 0) {
    TB_CUDA(cudaMemsetAsync(out, 0, sizeof(double), stream));
    return;
  }
  k_dot_partial<<<kRedBlocks, kThreads, 0, stream>>>(x, y, n, part);
  k_dot_final<<<1, 1024, 0, stream>>>(part, kRedBlocks, out, scale, root);
  TB_CUDA(cudaGetLastError());
}

void launch_denom(double* t, const double* r, double scale, const DenomBlock* blocks, const DenomUnit* units,
                  int nunits, int nmodes, const double* eps, DenomSigns signs, cudaStream_t stream) {
  if(nunits <= 0) return;
  k_denom<false><<<denom_grid<false>(nunits), kThreads, 0, stream>>>(t, r, scale, blocks, units, nunits, nmodes, eps,
                                                                    signs, nullptr);
  TB_CUDA(cudaGetLastError());
}

void launch_fill_random(double* x, int64_t n, uint64_t seed, uint64_t first, int dist, double p0,
                        double p1, cudaStream_t stream) {
  if(n <= 0) return;
  k_fill_random<<<grid_for(n, 4), kThreads, 0, stream>>>(x, n, host_splitmix64(seed), first, dist,
                                                         p0, p1);
  TB_CUDA(cudaGetLastError());
}

} // namespace tb
