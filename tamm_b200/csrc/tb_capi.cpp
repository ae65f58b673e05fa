// extern "C" entry points of libtamm_b200.so (declared in include/tamm_b200.h).
// Every entry converts library exceptions into a status code + tb_last_error().
#include "tb_runtime.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

namespace tb {
const std::string&   last_error();
std::shared_ptr<TIS> make_tis(const std::shared_ptr<IndexSpace>& is, int64_t tile,
                              const int64_t* tiles, int64_t ntiles);
std::shared_ptr<TIS> tis_named(const TIS& parent, const std::string& name);
std::shared_ptr<TIS> tis_subrange(const TIS& parent, int64_t first, int64_t last);
std::shared_ptr<WorkList> mult_worklist(const Op& op, const LabelClasses& lc, bool upload, int rank = 0,
                                        int nranks = 1);
void set_read_only(Tensor& T, bool on);

// Mode dispatch of one grouped contraction.
void run_contract(Plan& plan, const WorkList& wl, double alpha, const double* A, const double* B,
                  double* C, cudaStream_t stream, Arena* arena) {
  plan.last          = tb_stats{};
  plan.last.flops     = wl.flops;
  plan.last.flops_run = wl.flops_run;
  plan.last.mode      = plan.mode;
  plan.last.tile_n   = plan.tile_n;
  plan.arena      = arena;
  if(wl.tasks.empty()) return;
  switch(plan.mode) {
    case TB_MODE_FP64:
      if(plan.profile) {
        cudaEvent_t e0, e1;
        TB_CUDA(cudaEventCreate(&e0));
        TB_CUDA(cudaEventCreate(&e1));
        TB_CUDA(cudaEventRecord(e0, stream));
        launch_contract_fp64(plan, wl, alpha, 1.0, plan.store ? 1 : 0, A, B, C, stream);
        TB_CUDA(cudaEventRecord(e1, stream));
        TB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        TB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        plan.last.gemm_ms = ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
      }
      else launch_contract_fp64(plan, wl, alpha, 1.0, plan.store ? 1 : 0, A, B, C, stream);
      break;
    case TB_MODE_INT8: contract_int8(plan, wl, alpha, A, B, C, stream); break;
    case TB_MODE_BF16X3: contract_bf16x3(plan, wl, alpha, A, B, C, stream); break;
    default: fail(TB_ERR_INVALID, "unknown precision mode");
  }
}
} // namespace tb

using namespace tb;

#include "tb_api.hpp"

namespace tb {
Labeled labeled_from_c(const tb_labeled& x) {
  TB_EXPECTS(x.tensor != nullptr, "labelled operand without a tensor");
  Labeled l;
  l.t = x.tensor->p.get();
  for(int i = 0; i < l.t->nmodes; i++) {
    TB_EXPECTS(x.labels != nullptr, "labelled operand without labels");
    l.labels.push_back(x.labels[i]);
    l.ltis.push_back((x.label_tis && x.label_tis[i]) ? x.label_tis[i]->p : l.t->tis[i]);
  }
  return l;
}

} // namespace tb

#define REQUIRE_ARG(x) TB_EXPECTS((x), #x " must be non-null / valid")

extern "C" {

const char* tb_status_string(int s) {
  switch(s) {
    case TB_OK: return "ok";
    case TB_ERR_INVALID: return "invalid argument";
    case TB_ERR_NOT_IMPLEMENTED: return "not implemented";
    case TB_ERR_NO_MEMORY: return "out of memory";
    case TB_ERR_CUDA: return "CUDA error";
    case TB_ERR_TIMEOUT: return "device wait timed out";
    case TB_ERR_DEVICE: return "device error flag raised";
    case TB_ERR_STATE: return "invalid state";
    default: return "unknown status";
  }
}

int tb_last_error(char* buf, size_t len) {
  if(buf == nullptr || len == 0) return TB_ERR_INVALID;
  const std::string& m = tb::last_error();
  std::strncpy(buf, m.c_str(), len - 1);
  buf[len - 1] = '\0';
  return TB_OK;
}

int tb_version(int* major, int* minor) {
  if(major) *major = 0;
  if(minor) *minor = 1;
  return TB_OK;
}

// ---------------------------------------------------------------- kernel tier

int tb_block_multiply(double alpha, const double* a, const int64_t* adims, const int* alabels,
                      int na, const double* b, const int64_t* bdims, const int* blabels, int nb,
                      double beta, double* c, const int64_t* cdims, const int* clabels, int nc,
                      int is_assign, int mode, void* stream) {
  TB_API_BEGIN
  REQUIRE_ARG(a != nullptr && b != nullptr && c != nullptr); // multiply.hpp:226
  TB_EXPECTS((na == 0 || (adims && alabels)) && (nb == 0 || (bdims && blabels)) &&
               (nc == 0 || (cdims && clabels)),
             "dims/labels arrays must be given for every non-scalar operand");
  Plan plan;
  plan.lc   = classify(clabels, nc, alabels, na, blabels, nb);
  plan.mode = mode;
  std::unique_ptr<WorkList> wl(single_block_worklist(plan.lc, adims, bdims, cdims));
  auto st = static_cast<cudaStream_t>(stream);
  WorkList& w = *wl;
  finalize_worklist(plan.lc, w);
  if(mode == TB_MODE_FP64 || plan.lc.nar > 0 || plan.lc.nbr > 0) {
    // A-only / B-only reduction steps are beta-chained on the FP64 tensor-core path.
    launch_contract_fp64(plan, w, alpha, beta, is_assign, a, b, c, st);
  }
  else {
    if(is_assign) launch_fill(c, [&] {
        int64_t n = 1;
        for(int i = 0; i < nc; i++) n *= cdims[i];
        return n;
      }(), 0.0, 1, st);
    run_contract(plan, w, alpha, a, b, c, st, nullptr);
  }
  TB_CUDA(cudaStreamSynchronize(st)); // the work list is released on return
  TB_API_END
}

int tb_block_assign(double* dst, const int64_t* ddims, const int* dlabels, int nd, double scale,
                    const double* src, const int64_t* sdims, const int* slabels, int ns,
                    int is_assign, void* stream) {
  TB_API_BEGIN
  REQUIRE_ARG(dst != nullptr && src != nullptr);
  TB_EXPECTS((nd == 0 || (ddims && dlabels)) && (ns == 0 || (sdims && slabels)),
             "dims/labels arrays must be given for every non-scalar operand");
  AssignLoop lp = plan_assign(ddims, dlabels, nd, sdims, slabels, ns);
  launch_assign(lp, dst, scale, src, is_assign, static_cast<cudaStream_t>(stream));
  TB_API_END
}

int tb_fill(double* x, int64_t n, double value, int is_assign, void* stream) {
  TB_API_BEGIN
  REQUIRE_ARG(x != nullptr || n == 0);
  TB_EXPECTS(n >= 0, "negative length");
  launch_fill(x, n, value, is_assign, static_cast<cudaStream_t>(stream));
  TB_API_END
}

int tb_axpby(double alpha, const double* x, double beta, double* y, int64_t n, void* stream) {
  TB_API_BEGIN
  REQUIRE_ARG((x != nullptr && y != nullptr) || n == 0);
  TB_EXPECTS(n >= 0, "negative length");
  launch_axpby(alpha, x, beta, y, n, static_cast<cudaStream_t>(stream));
  TB_API_END
}

int tb_norm2(const double* x, int64_t n, double* host_out, void* stream) {
  TB_API_BEGIN
  REQUIRE_ARG(host_out != nullptr && (x != nullptr || n == 0));
  TB_EXPECTS(n >= 0, "negative length");
  *host_out = std::sqrt(reduce_dot(x, nullptr, n, static_cast<cudaStream_t>(stream)));
  TB_API_END
}

int tb_dot(const double* x, const double* y, int64_t n, double* host_out, void* stream) {
  TB_API_BEGIN
  REQUIRE_ARG(host_out != nullptr && ((x != nullptr && y != nullptr) || n == 0));
  TB_EXPECTS(n >= 0, "negative length");
  *host_out = reduce_dot(x, y, n, static_cast<cudaStream_t>(stream));
  TB_API_END
}

int tb_fill_random(double* x, int64_t n, uint64_t seed, uint64_t first, int dist, double p0,
                   double p1, void* stream) {
  TB_API_BEGIN
  REQUIRE_ARG(x != nullptr || n == 0);
  TB_EXPECTS(dist == 0 || dist == 1, "dist must be 0 (uniform) or 1 (normal)");
  launch_fill_random(x, n, seed, first, dist, p0, p1, static_cast<cudaStream_t>(stream));
  TB_API_END
}

int tb_plan_contraction(const int* clabels, int nc, const int* alabels, int na, const int* blabels,
                        int nb, int mode, double err_target, int nslices, tb_plan* out) {
  TB_API_BEGIN
  REQUIRE_ARG(out != nullptr);
  TB_EXPECTS(mode == TB_MODE_FP64 || mode == TB_MODE_INT8 || mode == TB_MODE_BF16X3,
             "unknown precision mode");
  TB_EXPECTS(nslices == 0 || (nslices >= 2 && nslices <= 8), "nslices must be 0 or 2..8");
  auto* p         = new tb_plan_s();
  p->p.lc         = classify(clabels, nc, alabels, na, blabels, nb);
  p->p.mode       = mode;
  p->p.err_target = err_target > 0 ? err_target : 1e-11;
  p->p.nslices    = nslices;
  *out            = p;
  TB_API_END
}

int tb_plan_destroy(tb_plan plan) {
  delete plan;
  return TB_OK;
}

int tb_worklist_build(tb_plan plan, int64_t ngroups, const int64_t* group_c_off,
                      const int32_t* group_cdims, const int64_t* group_task_begin,
                      const int64_t* task_a_off, const int64_t* task_b_off,
                      const int32_t* task_adims, const int32_t* task_bdims, tb_worklist* out) {
  TB_API_BEGIN
  REQUIRE_ARG(plan != nullptr && out != nullptr && ngroups >= 0);
  REQUIRE_ARG(ngroups == 0 || (group_c_off && group_task_begin));
  const LabelClasses& lc = plan->p.lc;
  auto                wl = std::make_unique<WorkList>();
  const int64_t       nt = ngroups > 0 ? group_task_begin[ngroups] : 0;
  TB_EXPECTS(nt >= 0 && nt < (1ll << 31), "task count out of range");
  TB_EXPECTS(nt == 0 || (task_a_off && task_b_off && (lc.na == 0 || task_adims) &&
                         (lc.nb == 0 || task_bdims)),
             "task arrays must be given");
  wl->groups.resize(ngroups);
  for(int64_t g = 0; g < ngroups; g++) {
    DevGroup& d = wl->groups[g];
    d.c_off     = group_c_off[g];
    TB_EXPECTS(group_task_begin[g] <= group_task_begin[g + 1], "task ranges must be ascending");
    d.task_begin = (int32_t) group_task_begin[g];
    d.task_end   = (int32_t) group_task_begin[g + 1];
    for(int i = 0; i < lc.nc; i++) d.cdims[i] = group_cdims[g * lc.nc + i];
  }
  wl->tasks.resize(nt);
  for(int64_t t = 0; t < nt; t++) {
    DevTask& d = wl->tasks[t];
    d.a_off    = task_a_off[t];
    d.b_off    = task_b_off[t];
    for(int i = 0; i < lc.na; i++) d.adims[i] = task_adims[t * lc.na + i];
    for(int i = 0; i < lc.nb; i++) d.bdims[i] = task_bdims[t * lc.nb + i];
  }
  finalize_worklist(lc, *wl);
  auto* h = new tb_worklist_s();
  h->p    = std::move(wl);
  *out    = h;
  TB_API_END
}

int tb_worklist_destroy(tb_worklist wl) {
  delete wl;
  return TB_OK;
}

int tb_worklist_info(tb_worklist wl, int64_t* ntasks, double* flops) {
  TB_API_BEGIN
  REQUIRE_ARG(wl != nullptr);
  if(ntasks) *ntasks = (int64_t) wl->p->tasks.size();
  if(flops) *flops = wl->p->flops;
  TB_API_END
}

int tb_contract(tb_plan plan, tb_worklist wl, double alpha, const double* a, const double* b,
                double* c, void* stream) {
  TB_API_BEGIN
  REQUIRE_ARG(plan != nullptr && wl != nullptr);
  REQUIRE_ARG(a != nullptr && b != nullptr && c != nullptr);
  run_contract(plan->p, *wl->p, alpha, a, b, c, static_cast<cudaStream_t>(stream), nullptr);
  TB_API_END
}

int tb_plan_stats(tb_plan plan, tb_stats* out) {
  TB_API_BEGIN
  REQUIRE_ARG(plan != nullptr && out != nullptr);
  *out = plan->p.last;
  TB_API_END
}

// --------------------------------------------------------------- runtime tier

int tb_ctx_create(int device, int64_t pool_bytes, tb_ctx* out) {
  TB_API_BEGIN
  REQUIRE_ARG(out != nullptr);
  int ndev = 0;
  TB_CUDA(cudaGetDeviceCount(&ndev));
  TB_EXPECTS(device >= 0 && device < ndev, "device index out of range");
  TB_CUDA(cudaSetDevice(device));
  auto ctx    = std::make_unique<Ctx>();
  ctx->device = device;
  TB_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  if(pool_bytes <= 0) { // TAMM_GPU_POOL default: 80% of free memory
    size_t fr = 0, tot = 0;
    TB_CUDA(cudaMemGetInfo(&fr, &tot));
    pool_bytes = (int64_t) (0.8 * (double) fr);
  }
  ctx->arena = std::make_unique<Arena>(device, pool_bytes);
  auto* h    = new tb_ctx_s();
  h->p       = std::move(ctx);
  *out       = h;
  TB_API_END
}

int tb_ctx_destroy(tb_ctx ctx) {
  delete ctx;
  return TB_OK;
}

int tb_ctx_set_precision(tb_ctx ctx, int mode, double err_target, int nslices) {
  TB_API_BEGIN
  REQUIRE_ARG(ctx != nullptr);
  TB_EXPECTS(mode == TB_MODE_FP64 || mode == TB_MODE_INT8 || mode == TB_MODE_BF16X3,
             "unknown precision mode");
  TB_EXPECTS(nslices == 0 || (nslices >= 2 && nslices <= 8), "nslices must be 0 or 2..8");
  ctx->p->mode       = mode;
  ctx->p->err_target = err_target > 0 ? err_target : 1e-11;
  ctx->p->nslices    = nslices;
  TB_API_END
}

int tb_ctx_set_digit_cache(tb_ctx ctx, int64_t bytes) {
  TB_API_BEGIN
  REQUIRE_ARG(ctx != nullptr);
  TB_EXPECTS(bytes >= 0, "negative cache size");
  ctx->p->digit_cache_bytes = bytes;
  TB_API_END
}

int tb_ctx_digit_cache_info(tb_ctx ctx, int64_t* used, int64_t* limit) {
  TB_API_BEGIN
  REQUIRE_ARG(ctx != nullptr);
  if(used) *used = ctx->p->digit_cache_used;
  if(limit) *limit = ctx->p->digit_cache_bytes;
  TB_API_END
}

int tb_ctx_stream(tb_ctx ctx, void** stream) {
  TB_API_BEGIN
  REQUIRE_ARG(ctx != nullptr && stream != nullptr);
  *stream = ctx->p->stream;
  TB_API_END
}

int tb_ctx_synchronize(tb_ctx ctx) {
  TB_API_BEGIN
  REQUIRE_ARG(ctx != nullptr);
  TB_CUDA(cudaSetDevice(ctx->p->device));
  TB_CUDA(cudaStreamSynchronize(ctx->p->stream));
  if(ctx->p->h2d) TB_CUDA(cudaStreamSynchronize(ctx->p->h2d));
  if(ctx->p->d2h) TB_CUDA(cudaStreamSynchronize(ctx->p->d2h));
  TB_API_END
}

int tb_ctx_alloc(tb_ctx ctx, int64_t bytes, void** out) {
  TB_API_BEGIN
  REQUIRE_ARG(ctx != nullptr && out != nullptr);
  TB_EXPECTS(bytes >= 0, "negative allocation size");
  *out = ctx->p->arena->allocate(std::max<int64_t>(bytes, 1));
  TB_API_END
}

int tb_ctx_free(tb_ctx ctx, void* p) {
  TB_API_BEGIN
  REQUIRE_ARG(ctx != nullptr);
  if(p) ctx->p->arena->deallocate(p);
  TB_API_END
}

int tb_ctx_join(tb_ctx ctx) {
  TB_API_BEGIN
  REQUIRE_ARG(ctx != nullptr);
  Ctx& c = *ctx->p;
  TB_CUDA(cudaSetDevice(c.device));
  for(cudaStream_t x: {c.h2d, c.d2h}) {
    if(!x) continue;
    cudaEvent_t e;
    TB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    TB_CUDA(cudaEventRecord(e, x));
    TB_CUDA(cudaStreamWaitEvent(c.stream, e, 0));
    TB_CUDA(cudaEventDestroy(e)); // released once the wait is resolved
  }
  TB_API_END
}

int tb_ctx_arena_info(tb_ctx ctx, int64_t* used, int64_t* peak, int64_t* capacity) {
  TB_API_BEGIN
  REQUIRE_ARG(ctx != nullptr);
  if(used) *used = ctx->p->arena->used();
  if(peak) *peak = ctx->p->arena->peak();
  if(capacity) *capacity = ctx->p->arena->capacity();
  TB_API_END
}

int tb_is_create(int64_t n, int nnamed, const char* const* names, const int* name_nranges,
                 const int64_t* name_ranges, int nspin, const int* spin_values,
                 const int* spin_nranges, const int64_t* spin_ranges, tb_is* out) {
  TB_API_BEGIN
  REQUIRE_ARG(out != nullptr && n >= 0 && nnamed >= 0 && nspin >= 0);
  auto is = std::make_shared<IndexSpace>();
  is->n   = n;
  int64_t r = 0;
  for(int i = 0; i < nnamed; i++) {
    REQUIRE_ARG(names && names[i] && name_nranges);
    std::vector<Range> rs;
    for(int k = 0; k < name_nranges[i]; k++, r++) {
      const int64_t lo = name_ranges[2 * r], hi = name_ranges[2 * r + 1];
      TB_EXPECTS(lo >= 0 && lo <= hi && hi <= n, "named range out of bounds");
      rs.push_back({lo, hi});
    }
    is->named.push_back({names[i], rs});
  }
  r = 0;
  for(int i = 0; i < nspin; i++) {
    REQUIRE_ARG(spin_values && spin_nranges);
    std::vector<Range> rs;
    for(int k = 0; k < spin_nranges[i]; k++, r++) {
      const int64_t lo = spin_ranges[2 * r], hi = spin_ranges[2 * r + 1];
      TB_EXPECTS(lo >= 0 && lo <= hi && hi <= n, "spin range out of bounds");
      rs.push_back({lo, hi});
    }
    is->spin.push_back({spin_values[i], rs});
  }
  auto* h = new tb_is_s();
  h->p    = is;
  *out    = h;
  TB_API_END
}

int tb_is_destroy(tb_is is) {
  delete is;
  return TB_OK;
}

int tb_tis_create(tb_is is, int64_t tile, const int64_t* tiles, int64_t ntiles, tb_tis* out) {
  TB_API_BEGIN
  REQUIRE_ARG(is != nullptr && out != nullptr);
  auto t  = make_tis(is->p, tile, tiles, ntiles);
  auto* h = new tb_tis_s();
  h->p    = t;
  *out    = h;
  TB_API_END
}

int tb_tis_named(tb_tis tis, const char* name, tb_tis* out) {
  TB_API_BEGIN
  REQUIRE_ARG(tis != nullptr && name != nullptr && out != nullptr);
  auto* h = new tb_tis_s();
  h->p    = tis_named(*tis->p, name);
  *out    = h;
  TB_API_END
}

int tb_tis_subrange(tb_tis tis, int64_t first_tile, int64_t last_tile, tb_tis* out) {
  TB_API_BEGIN
  REQUIRE_ARG(tis != nullptr && out != nullptr);
  auto* h = new tb_tis_s();
  h->p    = tis_subrange(*tis->p, first_tile, last_tile);
  *out    = h;
  TB_API_END
}

int tb_tis_num_tiles(tb_tis tis, int64_t* ntiles) {
  TB_API_BEGIN
  REQUIRE_ARG(tis != nullptr && ntiles != nullptr);
  *ntiles = tis->p->ntiles();
  TB_API_END
}

int tb_tis_tiles(tb_tis tis, int64_t* sizes, int* spins, int64_t* root_tiles) {
  TB_API_BEGIN
  REQUIRE_ARG(tis != nullptr);
  for(int64_t t = 0; t < tis->p->ntiles(); t++) {
    if(sizes) sizes[t] = tis->p->size(t);
    if(spins) spins[t] = tis->p->spin(t);
    if(root_tiles) root_tiles[t] = tis->p->tiles[t];
  }
  TB_API_END
}

int tb_tis_destroy(tb_tis tis) {
  delete tis;
  return TB_OK;
}

static tb_tensor new_tensor(int nmodes, const tb_tis* tis, const int* mask, const int* dep_modes = nullptr);

int tb_tis_create_dependent(tb_tis reference, int ndep, const tb_tis* on, int64_t nkeys, const int64_t* keys,
                            const tb_tis* values, tb_tis* out) {
  TB_API_BEGIN
  REQUIRE_ARG(reference != nullptr && out != nullptr && on != nullptr && ndep >= 1 && ndep <= 4);
  REQUIRE_ARG(nkeys >= 0 && (nkeys == 0 || (keys != nullptr && values != nullptr)));
  TB_EXPECTS(!reference->p->dep, "the reference of a dependent space must not be dependent itself");
  auto dep = std::make_shared<Dependency>();
  for(int k = 0; k < ndep; k++) {
    REQUIRE_ARG(on[k] != nullptr);
    dep->on.push_back(on[k]->p);
  }
  const TIS& ref = *reference->p;
  for(int64_t n = 0; n < nkeys; n++) {
    std::vector<int64_t> key(keys + n * ndep, keys + (n + 1) * ndep);
    for(int k = 0; k < ndep; k++)
      TB_EXPECTS(key[k] >= 0 && key[k] < dep->on[k]->ntiles(), "dependency key tile out of range");
    REQUIRE_ARG(values[n] != nullptr);
    const TIS& val = *values[n]->p;
    TB_EXPECTS(val.root == ref.root, "a dependent space's tiles must be tiles of its reference space");
    std::vector<uint8_t> ok(ref.ntiles(), 0);
    for(int64_t t: val.tiles) {
      const int64_t x = ref.find_root(t);
      TB_EXPECTS(x >= 0, "a dependent space's tiles must be tiles of its reference space");
      ok[x] = 1;
    }
    TB_EXPECTS(dep->valid.emplace(key, ok).second, "dependency key listed twice");
  }
  auto* h  = new tb_tis_s();
  h->p     = std::make_shared<TIS>();
  h->p->root  = ref.root;
  h->p->tiles = ref.tiles;
  h->p->dep   = dep;
  *out        = h;
  TB_API_END
}

int tb_tensor_create_dependent(int nmodes, const tb_tis* tis, const int* spin_mask, const int* dep_modes,
                               tb_tensor* out) {
  TB_API_BEGIN
  REQUIRE_ARG(out != nullptr && dep_modes != nullptr);
  *out = new_tensor(nmodes, tis, spin_mask, dep_modes);
  TB_API_END
}

static tb_tensor new_tensor(int nmodes, const tb_tis* tis, const int* mask, const int* dep_modes) {
  TB_EXPECTS(nmodes >= 0 && nmodes <= kMaxModes, "tensor rank out of range (max 8)");
  auto t      = std::make_unique<Tensor>();
  t->nmodes   = nmodes;
  t->has_spin = mask != nullptr;
  for(int i = 0; i < nmodes; i++) {
    REQUIRE_ARG(tis != nullptr && tis[i] != nullptr);
    t->tis.push_back(tis[i]->p);
    if(mask) {
      TB_EXPECTS(mask[i] >= 0 && mask[i] <= 2, "spin mask entries are 0 upper, 1 lower, 2 ignore");
      t->mask[i] = mask[i];
    }
  }
  t->dep_modes.assign(nmodes, {});
  for(int i = 0; i < nmodes; i++) {
    const auto& d = t->tis[i]->dep;
    if(!d) continue;
    TB_EXPECTS(dep_modes != nullptr, "a mode over a dependent space needs the modes it depends on "
                                     "(tb_tensor_create_dependent)");
    for(int k = 0; k < (int) d->on.size(); k++) {
      const int o = dep_modes[4 * i + k];
      TB_EXPECTS(o >= 0 && o < nmodes && o != i, "dependent mode refers to a mode out of range");
      TB_EXPECTS(!t->tis[o]->dep, "a dependent mode must depend on ordinary modes");
      TB_EXPECTS(t->tis[o]->root == d->on[k]->root, "a dependent mode's key mode is not over the space it depends on");
      t->dep_modes[i].push_back(o);
    }
  }
  t->build_table();
  auto* h = new tb_tensor_s();
  h->p    = std::move(t);
  return h;
}

int tb_tensor_create(int nmodes, const tb_tis* tis, const int* spin_mask, tb_tensor* out) {
  TB_API_BEGIN
  REQUIRE_ARG(out != nullptr);
  *out = new_tensor(nmodes, tis, spin_mask);
  TB_API_END
}

int tb_tensor_create_lambda(int nmodes, const tb_tis* tis, const int* spin_mask, tb_block_fn fn, void* user,
                            tb_tensor* out) {
  TB_API_BEGIN
  REQUIRE_ARG(out != nullptr && fn != nullptr);
  tb_tensor t          = new_tensor(nmodes, tis, spin_mask);
  t->p->lambda_block   = fn;
  t->p->lambda_user    = user;
  *out                 = t;
  TB_API_END
}

int tb_tensor_create_built(int nmodes, const tb_tis* tis, const int* spin_mask, tb_batch_fn fn, void* user,
                           tb_tensor* out) {
  TB_API_BEGIN
  REQUIRE_ARG(out != nullptr && fn != nullptr);
  tb_tensor t          = new_tensor(nmodes, tis, spin_mask);
  t->p->lambda_batch   = fn;
  t->p->lambda_user    = user;
  *out                 = t;
  TB_API_END
}

int tb_tensor_space(tb_tensor t, int mode, tb_tis* out) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && out != nullptr);
  TB_EXPECTS(mode >= 0 && mode < t->p->nmodes, "mode out of range");
  auto* h = new tb_tis_s();
  h->p    = t->p->tis[mode];
  *out    = h;
  TB_API_END
}

int tb_tensor_set_batch_bytes(tb_tensor t, int64_t bytes) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr);
  TB_EXPECTS(bytes >= 0, "negative batch size");
  t->p->batch_bytes = bytes;
  TB_API_END
}

int tb_tensor_create_spin_sizes(int nmodes, const tb_tis* tis, int nupper, int nlower,
                                tb_tensor* out) {
  TB_API_BEGIN
  REQUIRE_ARG(out != nullptr);
  // TensorImpl(TiledIndexSpaceVec, std::vector<size_t> spin_sizes) (tensor_impl.hpp:153-178)
  TB_EXPECTS(nupper >= 0 && nlower >= 0 && nupper + nlower <= nmodes,
             "spin sizes exceed the number of modes");
  int mask[kMaxModes];
  for(int i = 0; i < nmodes; i++) mask[i] = i < nupper ? 0 : (i < nupper + nlower ? 1 : 2);
  *out = new_tensor(nmodes, tis, mask);
  TB_API_END
}

int tb_tensor_allocate(tb_tensor t, tb_ctx ctx) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && ctx != nullptr);
  if(t->p->data != nullptr) fail(TB_ERR_STATE, "tensor already allocated");
  if(t->p->is_lambda()) fail(TB_ERR_STATE, "a lambda tensor has no storage of its own");
  TB_CUDA(cudaSetDevice(ctx->p->device));
  t->p->data = static_cast<double*>(ctx->p->arena->allocate(sizeof(double) * std::max<int64_t>(t->p->nelems, 1)));
  t->p->ctx  = ctx->p;
  TB_API_END
}

int tb_tensor_attach(tb_tensor t, tb_ctx ctx, void* device_ptr, int64_t bytes) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && ctx != nullptr && device_ptr != nullptr);
  if(t->p->data != nullptr) fail(TB_ERR_STATE, "tensor already allocated");
  TB_EXPECTS(bytes >= (int64_t) sizeof(double) * t->p->nelems, "attached storage smaller than the tensor");
  TB_EXPECTS((reinterpret_cast<uintptr_t>(device_ptr) & 15) == 0, "attached storage must be 16-byte aligned");
  t->p->data = static_cast<double*>(device_ptr);
  t->p->owns = false;
  t->p->ctx  = ctx->p;
  TB_API_END
}

int tb_tensor_deallocate(tb_tensor t) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr);
  if(t->p->data && t->p->ctx && t->p->owns) t->p->ctx->arena->deallocate(t->p->data);
  set_read_only(*t->p, false);
  t->p->data = nullptr;
  t->p->owns = true;
  t->p->ctx.reset();
  TB_API_END
}

int tb_tensor_destroy(tb_tensor t) {
  if(t == nullptr) return TB_OK;
  tb_tensor_deallocate(t);
  delete t;
  return TB_OK;
}

int tb_tensor_info(tb_tensor t, int* nmodes, int64_t* nblocks, int64_t* nelems) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr);
  if(nmodes) *nmodes = t->p->nmodes;
  if(nblocks) *nblocks = (int64_t) t->p->keys.size();
  if(nelems) *nelems = t->p->nelems;
  TB_API_END
}

int tb_tensor_block_table(tb_tensor t, int64_t* keys, int64_t* offsets) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr);
  if(keys) std::copy(t->p->keys.begin(), t->p->keys.end(), keys);
  if(offsets) std::copy(t->p->offsets.begin(), t->p->offsets.end(), offsets);
  TB_API_END
}

int tb_tensor_set_read_only(tb_tensor t, int on) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr);
  set_read_only(*t->p, on != 0);
  TB_API_END
}

int tb_tensor_read_only_info(tb_tensor t, int* on, int64_t* zero_blocks, int64_t* zero_elems) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr);
  const Tensor& T = *t->p;
  int64_t       nz = 0, ne = 0;
  for(size_t b = 0; b < T.zero_block.size(); b++)
    if(T.zero_block[b]) {
      nz++;
      ne += (b + 1 < T.keys.size() ? T.offsets[b + 1] : T.nelems) - T.offsets[b];
    }
  if(on) *on = T.read_only ? 1 : 0;
  if(zero_blocks) *zero_blocks = nz;
  if(zero_elems) *zero_elems = ne;
  TB_API_END
}

int tb_tensor_data(tb_tensor t, double** device_ptr) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && device_ptr != nullptr);
  *device_ptr = t->p->data;
  TB_API_END
}

int tb_tensor_is_non_zero(tb_tensor t, const int64_t* blockid, int* out) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && out != nullptr && (blockid != nullptr || t->p->nmodes == 0));
  t->p->check_blockid(blockid);
  *out = t->p->is_non_zero(blockid) ? 1 : 0;
  TB_API_END
}

int tb_tensor_block_size(tb_tensor t, const int64_t* blockid, int64_t* out) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && out != nullptr && (blockid != nullptr || t->p->nmodes == 0));
  t->p->check_blockid(blockid);
  *out = t->p->block_size(blockid);
  TB_API_END
}

int tb_tensor_block_dims(tb_tensor t, const int64_t* blockid, int64_t* dims) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && dims != nullptr && (blockid != nullptr || t->p->nmodes == 0));
  t->p->check_blockid(blockid);
  for(int i = 0; i < t->p->nmodes; i++) dims[i] = t->p->tis[i]->size(blockid[i]);
  TB_API_END
}

int tb_tensor_locate(tb_tensor t, const int64_t* blockid, int64_t* offset) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && offset != nullptr && (blockid != nullptr || t->p->nmodes == 0));
  t->p->check_blockid(blockid);
  *offset = t->p->locate(blockid);
  TB_API_END
}

static void block_io(tb_tensor t, const int64_t* blockid, double* host, int64_t n, int dir) {
  REQUIRE_ARG(t != nullptr && host != nullptr && (blockid != nullptr || t->p->nmodes == 0));
  Tensor& T = *t->p;
  T.check_blockid(blockid);
  const int64_t sz = T.block_size(blockid);
  TB_EXPECTS(n >= sz, "host buffer smaller than the block");
  if(dir != 0) T.require_writable();
  if(!T.is_non_zero(blockid)) { // tensor_impl.hpp:324-329 / :395 / :432
    if(dir == 0) std::fill(host, host + sz, 0.0);
    return;
  }
  T.require_allocated();
  TB_CUDA(cudaSetDevice(T.ctx->device));
  double* dptr = T.data + T.locate(blockid);
  if(dir == 0) {
    TB_CUDA(cudaMemcpyAsync(host, dptr, sizeof(double) * sz, cudaMemcpyDeviceToHost, T.ctx->stream));
    TB_CUDA(cudaStreamSynchronize(T.ctx->stream));
  }
  else if(dir == 1) {
    TB_CUDA(cudaMemcpyAsync(dptr, host, sizeof(double) * sz, cudaMemcpyHostToDevice, T.ctx->stream));
    TB_CUDA(cudaStreamSynchronize(T.ctx->stream));
  }
  else {
    double* tmp = static_cast<double*>(T.ctx->arena->allocate(sizeof(double) * sz));
    TB_CUDA(cudaMemcpyAsync(tmp, host, sizeof(double) * sz, cudaMemcpyHostToDevice, T.ctx->stream));
    launch_axpby(1.0, tmp, 1.0, dptr, sz, T.ctx->stream);
    TB_CUDA(cudaStreamSynchronize(T.ctx->stream));
    T.ctx->arena->deallocate(tmp);
  }
}

int tb_tensor_get(tb_tensor t, const int64_t* blockid, double* host, int64_t n) {
  TB_API_BEGIN
  block_io(t, blockid, host, n, 0);
  TB_API_END
}

int tb_tensor_put(tb_tensor t, const int64_t* blockid, const double* host, int64_t n) {
  TB_API_BEGIN
  block_io(t, blockid, const_cast<double*>(host), n, 1);
  TB_API_END
}

int tb_tensor_add(tb_tensor t, const int64_t* blockid, const double* host, int64_t n) {
  TB_API_BEGIN
  block_io(t, blockid, const_cast<double*>(host), n, 2);
  TB_API_END
}

int tb_tensor_write(tb_tensor t, const double* host, int64_t n) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && host != nullptr);
  TB_EXPECTS(n == t->p->nelems, "host buffer length must equal the stored element count");
  t->p->require_allocated();
  t->p->require_writable();
  TB_CUDA(cudaSetDevice(t->p->ctx->device));
  TB_CUDA(cudaMemcpyAsync(t->p->data, host, sizeof(double) * n, cudaMemcpyHostToDevice, t->p->ctx->stream));
  TB_CUDA(cudaStreamSynchronize(t->p->ctx->stream));
  TB_API_END
}

int tb_tensor_read(tb_tensor t, double* host, int64_t n) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && host != nullptr);
  TB_EXPECTS(n == t->p->nelems, "host buffer length must equal the stored element count");
  t->p->require_allocated();
  TB_CUDA(cudaSetDevice(t->p->ctx->device));
  TB_CUDA(cudaMemcpyAsync(host, t->p->data, sizeof(double) * n, cudaMemcpyDeviceToHost, t->p->ctx->stream));
  TB_CUDA(cudaStreamSynchronize(t->p->ctx->stream));
  TB_API_END
}

// Checkpoint file: header (magic, version, structure) + block keys + the packed store.
// The payload is the tensor's admitted blocks in row-major tile order, each block
// row-major: the element order of TAMM's tammio dataset (tamm_io.hpp:230-330, the
// file_offset of a block = sizes of the admitted blocks before it), without HDF5.
namespace {
constexpr char    kCkptMagic[8] = {'T', 'B', 'T', 'E', 'N', 'S', '0', '1'};
struct CkptFile {
  FILE* f = nullptr;
  ~CkptFile() {
    if(f) fclose(f);
  }
};
std::vector<int64_t> ckpt_structure(const Tensor& T) {
  std::vector<int64_t> h{T.nmodes, T.has_spin ? 1 : 0};
  for(int m = 0; m < T.nmodes; m++) {
    h.push_back(T.mask[m]);
    h.push_back(T.tis[m]->ntiles());
    for(int64_t x = 0; x < T.tis[m]->ntiles(); x++) {
      h.push_back(T.tis[m]->size(x));
      h.push_back(T.tis[m]->spin(x));
    }
  }
  h.push_back((int64_t) T.keys.size());
  h.push_back(T.nelems);
  return h;
}
} // namespace

int tb_tensor_save(tb_tensor t, const char* path) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && path != nullptr);
  const Tensor& T = *t->p;
  T.require_allocated();
  std::vector<double> host(std::max<int64_t>(T.nelems, 1));
  TB_CUDA(cudaSetDevice(T.ctx->device));
  TB_CUDA(cudaMemcpyAsync(host.data(), T.data, sizeof(double) * T.nelems, cudaMemcpyDeviceToHost, T.ctx->stream));
  TB_CUDA(cudaStreamSynchronize(T.ctx->stream));
  const std::vector<int64_t> h = ckpt_structure(T);
  const int64_t              nh = (int64_t) h.size();
  CkptFile                   cf;
  cf.f = fopen(path, "wb");
  TB_EXPECTS(cf.f != nullptr, std::string("cannot open for writing: ") + path);
  bool ok = fwrite(kCkptMagic, 1, 8, cf.f) == 8 && fwrite(&nh, 8, 1, cf.f) == 1 &&
            fwrite(h.data(), 8, h.size(), cf.f) == h.size() &&
            fwrite(T.keys.data(), 8, T.keys.size(), cf.f) == T.keys.size() &&
            (T.nelems == 0 || fwrite(host.data(), 8, T.nelems, cf.f) == (size_t) T.nelems);
  ok = (fclose(cf.f) == 0) && ok;
  cf.f = nullptr;
  TB_EXPECTS(ok, std::string("write failed: ") + path);
  TB_API_END
}

int tb_tensor_load(tb_tensor t, const char* path) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && path != nullptr);
  Tensor& T = *t->p;
  T.require_allocated();
  T.require_writable();
  CkptFile cf;
  cf.f = fopen(path, "rb");
  TB_EXPECTS(cf.f != nullptr, std::string("cannot open for reading: ") + path);
  char    magic[8];
  int64_t nh = 0;
  TB_EXPECTS(fread(magic, 1, 8, cf.f) == 8 && std::memcmp(magic, kCkptMagic, 8) == 0, "not a tensor checkpoint");
  TB_EXPECTS(fread(&nh, 8, 1, cf.f) == 1 && nh > 0 && nh < (1ll << 32), "corrupt checkpoint header");
  std::vector<int64_t> h(nh), keys;
  TB_EXPECTS(fread(h.data(), 8, h.size(), cf.f) == h.size(), "truncated checkpoint header");
  TB_EXPECTS(h == ckpt_structure(T), "checkpoint structure (spaces, tiles, spins, spin mask) differs from the tensor's");
  keys.resize(T.keys.size());
  TB_EXPECTS(fread(keys.data(), 8, keys.size(), cf.f) == keys.size() && keys == T.keys, "checkpoint block table differs");
  std::vector<double> host(std::max<int64_t>(T.nelems, 1));
  TB_EXPECTS(T.nelems == 0 || fread(host.data(), 8, T.nelems, cf.f) == (size_t) T.nelems, "truncated checkpoint data");
  TB_CUDA(cudaSetDevice(T.ctx->device));
  TB_CUDA(cudaMemcpyAsync(T.data, host.data(), sizeof(double) * T.nelems, cudaMemcpyHostToDevice, T.ctx->stream));
  TB_CUDA(cudaStreamSynchronize(T.ctx->stream));
  TB_API_END
}

// Asynchronous host transfers on the context's copy streams, ordered against the
// compute stream by events: a write waits until the compute work enqueued so far that
// touched the tensor is done, and later compute work waits for the write; a read
// waits for that compute work.  Host buffers must be pinned and stay untouched until
// tb_ctx_synchronize (or tb_sched_wait) returns.
int tb_tensor_write_async(tb_tensor t, const double* host, int64_t n) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && host != nullptr);
  Tensor& T = *t->p;
  TB_EXPECTS(n == T.nelems, "host buffer length must equal the stored element count");
  T.require_allocated();
  T.require_writable();
  Ctx& c = *T.ctx;
  TB_CUDA(cudaSetDevice(c.device));
  if(!c.h2d) TB_CUDA(cudaStreamCreateWithFlags(&c.h2d, cudaStreamNonBlocking));
  if(T.used) TB_CUDA(cudaStreamWaitEvent(c.h2d, T.used, 0));
  TB_CUDA(cudaMemcpyAsync(T.data, host, sizeof(double) * n, cudaMemcpyHostToDevice, c.h2d));
  if(!T.filled) TB_CUDA(cudaEventCreateWithFlags(&T.filled, cudaEventDisableTiming));
  TB_CUDA(cudaEventRecord(T.filled, c.h2d));
  TB_CUDA(cudaStreamWaitEvent(c.stream, T.filled, 0));
  TB_API_END
}

int tb_tensor_record_use(tb_tensor t) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr);
  Tensor& T = *t->p;
  T.require_allocated();
  TB_CUDA(cudaSetDevice(T.ctx->device));
  if(!T.used) TB_CUDA(cudaEventCreateWithFlags(&T.used, cudaEventDisableTiming));
  TB_CUDA(cudaEventRecord(T.used, T.ctx->stream));
  TB_API_END
}

int tb_tensor_read_async(tb_tensor t, double* host, int64_t n) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && host != nullptr);
  Tensor& T = *t->p;
  TB_EXPECTS(n == T.nelems, "host buffer length must equal the stored element count");
  T.require_allocated();
  Ctx& c = *T.ctx;
  TB_CUDA(cudaSetDevice(c.device));
  if(!c.d2h) TB_CUDA(cudaStreamCreateWithFlags(&c.d2h, cudaStreamNonBlocking));
  if(!T.used) { // nothing computed on it yet: order after everything enqueued so far
    TB_CUDA(cudaEventCreateWithFlags(&T.used, cudaEventDisableTiming));
    TB_CUDA(cudaEventRecord(T.used, c.stream));
  }
  TB_CUDA(cudaStreamWaitEvent(c.d2h, T.used, 0));
  if(T.filled) TB_CUDA(cudaStreamWaitEvent(c.d2h, T.filled, 0));
  TB_CUDA(cudaMemcpyAsync(host, T.data, sizeof(double) * n, cudaMemcpyDeviceToHost, c.d2h));
  TB_API_END
}

int tb_tensor_norm(tb_tensor t, double* out) {
  TB_API_BEGIN
  REQUIRE_ARG(t != nullptr && out != nullptr);
  t->p->require_allocated();
  TB_CUDA(cudaSetDevice(t->p->ctx->device));
  *out = std::sqrt(reduce_dot(t->p->data, nullptr, t->p->nelems, t->p->ctx->stream));
  TB_API_END
}

static Labeled to_labeled(const tb_labeled& x) { return tb::labeled_from_c(x); }

int tb_sched_create(tb_ctx ctx, tb_sched* out) {
  TB_API_BEGIN
  REQUIRE_ARG(ctx != nullptr && out != nullptr);
  auto* h   = new tb_sched_s();
  h->p      = std::make_unique<Sched>();
  h->p->ctx = ctx->p;
  *out      = h;
  TB_API_END
}

int tb_sched_destroy(tb_sched s) {
  delete s;
  return TB_OK;
}

int tb_sched_set(tb_sched s, tb_labeled lhs, double value, int is_assign) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  Op op;
  op.kind      = Op::Set;
  op.lhs       = to_labeled(lhs);
  op.value     = value;
  op.is_assign = is_assign;
  s->p->ops.push_back(op);
  TB_API_END
}

int tb_sched_add(tb_sched s, tb_labeled lhs, double alpha, tb_labeled rhs, int is_assign) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  Op op;
  op.kind      = Op::Add;
  op.lhs       = to_labeled(lhs);
  op.a         = to_labeled(rhs);
  op.alpha     = alpha;
  op.is_assign = is_assign;
  s->p->ops.push_back(op);
  TB_API_END
}

int tb_sched_mult_n(tb_sched s, tb_labeled lhs, double alpha, const tb_labeled* factors, int n, int is_assign) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr && factors != nullptr && n >= 1);
  std::vector<Labeled> f;
  for(int i = 0; i < n; i++) f.push_back(to_labeled(factors[i]));
  std::vector<Op> queued;
  queue_mult_n(*s->p, to_labeled(lhs), alpha, f, is_assign, [&](Op&& op) { queued.push_back(std::move(op)); });
  for(auto& op: queued) s->p->ops.push_back(std::move(op)); // all or nothing
  TB_API_END
}

int tb_opmin_order(tb_labeled lhs, const tb_labeled* factors, int n, int64_t* pairs, double* cost) {
  TB_API_BEGIN
  REQUIRE_ARG(factors != nullptr && n >= 1);
  std::vector<Labeled> f;
  for(int i = 0; i < n; i++) f.push_back(to_labeled(factors[i]));
  std::vector<int64_t> p;
  double               c = 0;
  mult_n_order(to_labeled(lhs), f, p, c);
  if(pairs) std::copy(p.begin(), p.end(), pairs);
  if(cost) *cost = c;
  TB_API_END
}

int tb_sched_map(tb_sched s, tb_labeled lhs, tb_labeled rhs, int fn, double p) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  TB_EXPECTS(fn >= TB_MAP_COPY && fn <= TB_MAP_ABS, "unknown element function (TB_MAP_*)");
  Op op;
  op.kind  = Op::Map;
  op.lhs   = to_labeled(lhs);
  op.a     = to_labeled(rhs);
  op.fn    = fn;
  op.value = p;
  if(op.lhs.labels != op.a.labels)
    fail(TB_ERR_NOT_IMPLEMENTED, "map: rhs must carry the lhs labels in the same order (no permutation)");
  s->p->ops.push_back(op);
  TB_API_END
}

int tb_sched_mult(tb_sched s, tb_labeled lhs, double alpha, tb_labeled a, tb_labeled b,
                  int is_assign) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  Op op;
  op.kind  = Op::Mult;
  op.lhs   = to_labeled(lhs);
  op.a     = to_labeled(a);
  op.b     = to_labeled(b);
  op.alpha = alpha;
  // validate the label classes now so a bad op fails at enqueue time
  (void) classify(op.lhs.labels.data(), (int) op.lhs.labels.size(), op.a.labels.data(),
                  (int) op.a.labels.size(), op.b.labels.data(), (int) op.b.labels.size());
  if(is_assign) { // MultOp::canonicalize (multop.hpp:255-269)
    Op set;
    set.kind      = Op::Set;
    set.lhs       = op.lhs;
    set.value     = 0.0;
    set.is_assign = 1;
    s->p->ops.push_back(set);
  }
  s->p->ops.push_back(op);
  TB_API_END
}

int tb_mult_info(tb_labeled lhs, tb_labeled a, tb_labeled b, int64_t* ngroups, int64_t* ntasks,
                 double* flops) {
  TB_API_BEGIN
  Op op;
  op.kind    = Op::Mult;
  op.lhs     = to_labeled(lhs);
  op.a       = to_labeled(a);
  op.b       = to_labeled(b);
  auto lc    = classify(op.lhs.labels.data(), (int) op.lhs.labels.size(), op.a.labels.data(),
                        (int) op.a.labels.size(), op.b.labels.data(), (int) op.b.labels.size());
  auto wl    = mult_worklist(op, lc, false);
  if(ngroups) *ngroups = (int64_t) wl->groups.size();
  if(ntasks) *ntasks = (int64_t) wl->tasks.size() + wl->ntasks_skipped;
  if(flops) *flops = wl->flops;
  TB_API_END
}

int tb_sched_set_owner(tb_sched s, int rank, int nranks) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  TB_EXPECTS(nranks >= 1 && rank >= 0 && rank < nranks, "rank must lie in [0, nranks)");
  s->p->rank   = rank;
  s->p->nranks = nranks;
  TB_API_END
}

int tb_mult_owned(tb_labeled lhs, tb_labeled a, tb_labeled b, int rank, int nranks, int64_t* ngroups,
                  double* flops, int64_t* c_offsets, int64_t cap) {
  TB_API_BEGIN
  TB_EXPECTS(nranks >= 1 && rank >= 0 && rank < nranks, "rank must lie in [0, nranks)");
  Op op;
  op.kind = Op::Mult;
  op.lhs  = to_labeled(lhs);
  op.a    = to_labeled(a);
  op.b    = to_labeled(b);
  auto lc = classify(op.lhs.labels.data(), (int) op.lhs.labels.size(), op.a.labels.data(),
                     (int) op.a.labels.size(), op.b.labels.data(), (int) op.b.labels.size());
  auto wl = mult_worklist(op, lc, false, rank, nranks);
  if(ngroups) *ngroups = (int64_t) wl->groups.size();
  if(flops) *flops = wl->flops;
  for(size_t g = 0; c_offsets && g < wl->groups.size() && (int64_t) g < cap; g++) c_offsets[g] = wl->groups[g].c_off;
  TB_API_END
}

int tb_sched_execute(tb_sched s, int hw, int profile) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  TB_EXPECTS(hw >= 0 && hw <= 2, "hw must be 0 (DEFAULT), 1 (CPU) or 2 (GPU)");
  s->p->execute(profile != 0);
  TB_CUDA(cudaStreamSynchronize(s->p->ctx->stream));
  TB_API_END
}

int tb_sched_execute_async(tb_sched s) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  s->p->deferred_checks = true;
  try {
    s->p->execute(false);
  } catch(...) {
    s->p->deferred_checks = false;
    throw;
  }
  s->p->deferred_checks = false;
  TB_API_END
}

int tb_sched_wait(tb_sched s) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  Ctx& c = *s->p->ctx;
  TB_CUDA(cudaSetDevice(c.device));
  TB_CUDA(cudaStreamSynchronize(c.stream));
  if(c.h2d) TB_CUDA(cudaStreamSynchronize(c.h2d));
  if(c.d2h) TB_CUDA(cudaStreamSynchronize(c.d2h));
  auto pending = std::move(s->p->pending);
  s->p->pending.clear();
  for(const auto& wl: pending) check_int8_errors(*wl, c.stream);
  TB_API_END
}

int tb_sched_profile(tb_sched s, int64_t* nops, double* ms, double* flops, int64_t cap) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  const int64_t n = (int64_t) s->p->prof_ms.size();
  if(nops) *nops = n;
  for(int64_t i = 0; i < n && i < cap; i++) {
    if(ms) ms[i] = s->p->prof_ms[i];
    if(flops) flops[i] = s->p->prof_flops[i];
  }
  TB_API_END
}

int tb_sched_op_stats(tb_sched s, int64_t index, tb_stats* out) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr && out != nullptr);
  TB_EXPECTS(index >= 0 && index < (int64_t) s->p->prof_stats.size(),
             "op index out of range (profile the execute first)");
  *out = s->p->prof_stats[index];
  TB_API_END
}

int tb_sched_dot(tb_sched s, int slot, double alpha, tb_labeled a, tb_labeled b) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  Op op;
  op.kind  = Op::Dot;
  op.a     = to_labeled(a);
  op.b     = to_labeled(b);
  op.alpha = alpha;
  op.slot  = slot;
  TB_EXPECTS(slot >= 0 && slot < Sched::kSlots, "scalar slot out of range (0..63)");
  TB_EXPECTS(op.a.labels == op.b.labels && op.a.t->keys == op.b.t->keys && op.a.t->offsets == op.b.t->offsets &&
               op.a.t->nmodes == op.b.t->nmodes,
             "dot operands need the same labels in the same order over the same block layout");
  s->p->ops.push_back(op);
  TB_API_END
}

int tb_sched_norm(tb_sched s, int slot, double alpha, tb_labeled a) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  Op op;
  op.kind  = Op::Dot;
  op.a     = to_labeled(a);
  op.b     = op.a;
  op.alpha = alpha;
  op.slot  = slot;
  op.root  = 1;
  TB_EXPECTS(slot >= 0 && slot < Sched::kSlots, "scalar slot out of range (0..63)");
  s->p->ops.push_back(op);
  TB_API_END
}

int tb_sched_scalars(tb_sched s, double* host, int n) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr && host != nullptr);
  TB_EXPECTS(n >= 0 && n <= Sched::kSlots, "at most 64 scalar slots");
  TB_CUDA(cudaSetDevice(s->p->ctx->device));
  TB_CUDA(cudaMemcpyAsync(host, s->p->scalars(), sizeof(double) * n, cudaMemcpyDeviceToHost, s->p->ctx->stream));
  TB_CUDA(cudaStreamSynchronize(s->p->ctx->stream));
  TB_API_END
}

int tb_sched_denom(tb_sched s, tb_labeled t, double alpha, tb_labeled r, const double* eps, int64_t neps,
                   const double* signs) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr && eps != nullptr && signs != nullptr && neps >= 0);
  Op op;
  op.kind  = Op::Denom;
  op.lhs   = to_labeled(t);
  op.a     = to_labeled(r);
  op.alpha = alpha;
  const Tensor& T = *op.lhs.t;
  TB_EXPECTS(T.nmodes >= 1, "denominator update of a scalar tensor");
  TB_EXPECTS(op.lhs.labels == op.a.labels && T.keys == op.a.t->keys && T.offsets == op.a.t->offsets,
             "denominator update: r needs t's labels and block layout");
  for(int m = 1; m < T.nmodes; m++)
    TB_EXPECTS(T.tis[m]->root->is == T.tis[0]->root->is, "denominator update: all modes over one root index space");
  auto d = std::make_shared<DenomSpec>();
  d->eps.assign(eps, eps + neps);
  for(int m = 0; m < T.nmodes; m++) d->signs[m] = signs[m];
  op.denom = d;
  s->p->ops.push_back(op);
  TB_API_END
}

int tb_sched_denom_energy(tb_sched s, int slot, double alpha, tb_labeled w, const double* eps, int64_t neps,
                          const double* signs) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr && eps != nullptr && signs != nullptr && neps >= 0);
  TB_EXPECTS(slot >= 0 && slot < Sched::kSlots, "scalar slot out of range (0..63)");
  Op op;
  op.kind  = Op::DenomEnergy;
  op.lhs   = to_labeled(w);
  op.alpha = alpha;
  op.slot  = slot;
  const Tensor& T = *op.lhs.t;
  TB_EXPECTS(T.nmodes >= 1, "denominator energy of a scalar tensor");
  for(int m = 1; m < T.nmodes; m++)
    TB_EXPECTS(T.tis[m]->root->is == T.tis[0]->root->is, "denominator energy: all modes over one root index space");
  auto d = std::make_shared<DenomSpec>();
  d->eps.assign(eps, eps + neps);
  for(int m = 0; m < T.nmodes; m++) d->signs[m] = signs[m];
  op.denom = d;
  s->p->ops.push_back(op);
  TB_API_END
}

int tb_sched_mult_energy(tb_sched s, int slot, double scale, tb_labeled lhs, double alpha, tb_labeled a,
                         tb_labeled b, const double* eps, int64_t neps, const double* signs) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr && eps != nullptr && signs != nullptr && neps >= 0);
  TB_EXPECTS(slot >= 0 && slot < Sched::kSlots, "scalar slot out of range (0..63)");
  Op op;
  op.kind   = Op::Mult;
  op.energy = true;
  op.lhs    = to_labeled(lhs);
  op.a      = to_labeled(a);
  op.b      = to_labeled(b);
  op.alpha  = alpha;
  op.slot   = slot;
  op.value  = scale;
  (void) classify(op.lhs.labels.data(), (int) op.lhs.labels.size(), op.a.labels.data(),
                  (int) op.a.labels.size(), op.b.labels.data(), (int) op.b.labels.size());
  const Tensor& T = *op.lhs.t;
  TB_EXPECTS(T.nmodes >= 1, "energy epilogue of a scalar output");
  for(int m = 1; m < T.nmodes; m++)
    TB_EXPECTS(T.tis[m]->root->is == T.tis[0]->root->is, "energy epilogue: all output modes over one root index space");
  auto d = std::make_shared<DenomSpec>();
  d->eps.assign(eps, eps + neps);
  for(int m = 0; m < T.nmodes; m++) d->signs[m] = signs[m];
  op.denom = d;
  s->p->ops.push_back(op);
  TB_API_END
}

int tb_sched_set_scalar(tb_sched s, int slot, double value) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  TB_EXPECTS(slot >= 0 && slot < Sched::kSlots, "scalar slot out of range (0..63)");
  Op op;
  op.kind  = Op::SetScalar;
  op.slot  = slot;
  op.value = value;
  s->p->ops.push_back(op);
  TB_API_END
}

int tb_sched_autotune(tb_sched s, int enable) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  s->p->autotune = enable != 0;
  TB_API_END
}

int tb_sched_tune_info(tb_sched s, int64_t index, int* mode, int* tile_n, int* ncand, int* cand_modes,
                       int* cand_tiles, double* cand_ms, int cap) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  const int64_t n0 = (int64_t) s->p->last_first;
  TB_EXPECTS(index >= 0 && n0 + index < (int64_t) s->p->start, "op index out of range (execute first)");
  const Op& op = s->p->ops[n0 + index];
  auto      it = s->p->tune_cache.find(op.tune_key);
  if(op.tune_key.empty() || it == s->p->tune_cache.end()) {
    if(ncand) *ncand = 0;
    return TB_OK;
  }
  const TuneChoice& c = it->second;
  if(mode) *mode = c.mode;
  if(tile_n) *tile_n = c.tile_n;
  if(ncand) *ncand = (int) c.ms.size();
  for(int i = 0; i < (int) c.ms.size() && i < cap; i++) {
    if(cand_modes) cand_modes[i] = c.modes[i];
    if(cand_tiles) cand_tiles[i] = c.tiles[i];
    if(cand_ms) cand_ms[i] = c.ms[i];
  }
  TB_API_END
}

int tb_sched_graph_create(tb_sched s, tb_graph* out) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr && out != nullptr);
  Sched& S = *s->p;
  TB_EXPECTS(S.start < S.ops.size(), "no queued ops to capture");
  S.execute(false); // warm-up: plans, work lists, split layouts, autotuner choices
  TB_CUDA(cudaStreamSynchronize(S.ctx->stream));
  const size_t first = S.last_first; // the warm-up ran ops [last_first, end)
  auto g = std::make_unique<Graph>();
  g->ctx        = S.ctx;
  g->pool.arena = S.ctx->arena.get();
  S.pinned      = &g->pool;
  cudaStream_t st = S.ctx->stream;
  TB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
  try {
    for(size_t i = first; i < S.ops.size(); i++) S.run(S.ops[i]);
  } catch(...) {
    cudaGraph_t dead = nullptr;
    cudaStreamEndCapture(st, &dead);
    if(dead) cudaGraphDestroy(dead);
    S.pinned = nullptr;
    throw;
  }
  S.pinned = nullptr;
  TB_CUDA(cudaStreamEndCapture(st, &g->graph));
  TB_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0));
  for(size_t i = first; i < S.ops.size(); i++)
    if(S.ops[i].kind == Op::Mult) {
      if(S.ops[i].wl) g->int8_lists.push_back(S.ops[i].wl);
      g->plans.push_back(S.ops[i].plan);
    }
  for(auto& wl: S.batch_lists) g->int8_lists.push_back(wl); // lambda batches
  S.batch_lists.clear();
  auto* h = new tb_graph_s();
  h->p    = std::move(g);
  *out    = h;
  TB_API_END
}

int tb_graph_launch(tb_graph g) {
  TB_API_BEGIN
  REQUIRE_ARG(g != nullptr);
  TB_CUDA(cudaSetDevice(g->p->ctx->device));
  TB_CUDA(cudaGraphLaunch(g->p->exec, g->p->ctx->stream));
  TB_API_END
}

int tb_graph_sync(tb_graph g) {
  TB_API_BEGIN
  REQUIRE_ARG(g != nullptr);
  TB_CUDA(cudaSetDevice(g->p->ctx->device));
  TB_CUDA(cudaStreamSynchronize(g->p->ctx->stream));
  for(const auto& wl: g->p->int8_lists) check_int8_errors(*wl, g->p->ctx->stream);
  TB_API_END
}

int tb_graph_destroy(tb_graph g) {
  delete g;
  return TB_OK;
}

int tb_sched_release(tb_sched s) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  TB_CUDA(cudaSetDevice(s->p->ctx->device));
  TB_CUDA(cudaStreamSynchronize(s->p->ctx->stream));
  s->p->ops.erase(s->p->ops.begin(), s->p->ops.begin() + (long) s->p->start);
  s->p->start = s->p->last_first = 0;
  s->p->plan_cache.clear();
  s->p->wl_cache.clear();
  s->p->fill_cache.clear();
  TB_API_END
}

int tb_sched_clear(tb_sched s) {
  TB_API_BEGIN
  REQUIRE_ARG(s != nullptr);
  s->p->ops.erase(s->p->ops.begin() + (long) s->p->start, s->p->ops.end());
  TB_API_END
}

} // extern "C"
