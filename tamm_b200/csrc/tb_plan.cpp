// Contraction planning: label classification (kernels::block_multiply's batch /
// outer / inner / reduce split) and device work lists.
#include "tb_internal.hpp"

#include <algorithm>
#include <cstring>
#include <mutex>
#include <sstream>

namespace tb {


namespace {
thread_local std::string g_last_error;

int find(const int* v, int n, int x) {
  for(int i = 0; i < n; i++)
    if(v[i] == x) return i;
  return -1;
}
} // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }
const std::string& last_error() { return g_last_error; }

[[noreturn]] void fail(int code, const std::string& msg) { throw Error(code, msg); }

LabelClasses classify(const int* cl, int nc, const int* al, int na, const int* bl, int nb) {
  TB_EXPECTS(nc >= 0 && nc <= kMaxModes && na >= 0 && na <= kMaxModes && nb >= 0 &&
               nb <= kMaxModes,
             "tensor rank out of range (max 8 modes)");
  for(int i = 0; i < nc; i++) TB_EXPECTS(find(cl, i, cl[i]) < 0, "repeated label in C");
  for(int i = 0; i < na; i++) TB_EXPECTS(find(al, i, al[i]) < 0, "repeated label in A");
  for(int i = 0; i < nb; i++) TB_EXPECTS(find(bl, i, bl[i]) < 0, "repeated label in B");
  LabelClasses lc;
  lc.nc = nc;
  lc.na = na;
  lc.nb = nb;
  auto room = [](int n, const char* what) {
    TB_EXPECTS(n < kMaxClass, std::string("more than 4 ") + what + " labels");
  };
  // multiply.hpp:238-260 — C labels in C order
  for(int i = 0; i < nc; i++) {
    const int pa = find(al, na, cl[i]), pb = find(bl, nb, cl[i]);
    if(pa >= 0 && pb >= 0) {
      room(lc.nbatch, "batch");
      lc.batch_c[lc.nbatch] = (int8_t) i;
      lc.batch_a[lc.nbatch] = (int8_t) pa;
      lc.batch_b[lc.nbatch] = (int8_t) pb;
      lc.nbatch++;
    }
    else if(pa >= 0) {
      room(lc.nm, "A-outer");
      lc.m_c[lc.nm] = (int8_t) i;
      lc.m_a[lc.nm] = (int8_t) pa;
      lc.nm++;
    }
    else if(pb >= 0) {
      room(lc.nn, "B-outer");
      lc.n_c[lc.nn] = (int8_t) i;
      lc.n_b[lc.nn] = (int8_t) pb;
      lc.nn++;
    }
    else
      fail(TB_ERR_INVALID, "EXPECTS failed: output label appears in neither input");
  }
  // multiply.hpp:262-282 — A labels in A order
  for(int i = 0; i < na; i++) {
    const int pb = find(bl, nb, al[i]), pc = find(cl, nc, al[i]);
    if(pb >= 0 && pc >= 0) continue;
    if(pb >= 0) {
      room(lc.nk, "inner");
      lc.k_a[lc.nk] = (int8_t) i;
      lc.k_b[lc.nk] = (int8_t) pb;
      lc.nk++;
    }
    else if(pc >= 0) continue;
    else {
      room(lc.nar, "A-only reduction");
      lc.ar_a[lc.nar++] = (int8_t) i;
    }
  }
  // multiply.hpp:284-302
  for(int i = 0; i < nb; i++) {
    const int pa = find(al, na, bl[i]), pc = find(cl, nc, bl[i]);
    if(pa < 0 && pc < 0) {
      room(lc.nbr, "B-only reduction");
      lc.br_b[lc.nbr++] = (int8_t) i;
    }
  }
  lc.a_contig = 2;
  if(na > 0) {
    for(int j = 0; j < lc.nm; j++)
      if(lc.m_a[j] == na - 1) lc.a_contig = 0;
    for(int j = 0; j < lc.nk; j++)
      if(lc.k_a[j] == na - 1) lc.a_contig = 1;
  }
  lc.b_contig = 2;
  if(nb > 0) {
    for(int j = 0; j < lc.nn; j++)
      if(lc.n_b[j] == nb - 1) lc.b_contig = 0;
    for(int j = 0; j < lc.nk; j++)
      if(lc.k_b[j] == nb - 1) lc.b_contig = 1;
  }
  return lc;
}

WorkList::~WorkList() {
  forget_int8_layout(this);
  if(d_groups || d_tasks || d_items) {
    int cur = -1;
    cudaGetDevice(&cur);
    if(device >= 0) cudaSetDevice(device);
    cudaFree(d_groups);
    cudaFree(d_tasks);
    cudaFree(d_items);
    if(cur >= 0) cudaSetDevice(cur);
  }
}

static void validate_task(const LabelClasses& lc, const DevGroup& g, const DevTask& t) {
  for(int j = 0; j < lc.nbatch; j++) {
    TB_EXPECTS(g.cdims[lc.batch_c[j]] == t.adims[lc.batch_a[j]] &&
                 g.cdims[lc.batch_c[j]] == t.bdims[lc.batch_b[j]],
               "batch label extents differ between C, A and B");
  }
  for(int j = 0; j < lc.nm; j++)
    TB_EXPECTS(g.cdims[lc.m_c[j]] == t.adims[lc.m_a[j]], "A-outer label extents differ (C vs A)");
  for(int j = 0; j < lc.nn; j++)
    TB_EXPECTS(g.cdims[lc.n_c[j]] == t.bdims[lc.n_b[j]], "B-outer label extents differ (C vs B)");
  for(int j = 0; j < lc.nk; j++)
    TB_EXPECTS(t.adims[lc.k_a[j]] == t.bdims[lc.k_b[j]], "inner label extents differ (A vs B)");
  int64_t asz = 1, bsz = 1, csz = 1;
  for(int i = 0; i < lc.na; i++) {
    TB_EXPECTS(t.adims[i] > 0, "block extent must be positive");
    asz *= t.adims[i];
  }
  for(int i = 0; i < lc.nb; i++) {
    TB_EXPECTS(t.bdims[i] > 0, "block extent must be positive");
    bsz *= t.bdims[i];
  }
  for(int i = 0; i < lc.nc; i++) csz *= g.cdims[i];
  TB_EXPECTS(asz < (1ll << 31) && bsz < (1ll << 31) && csz < (1ll << 31),
             "a single block must hold fewer than 2^31 elements");
  TB_EXPECTS(t.a_off >= 0 && t.b_off >= 0, "negative block offset");
}

double task_flops(const LabelClasses& lc, const DevGroup& g, const DevTask& t) {
  double csz = 1, k = 1;
  for(int i = 0; i < lc.nc; i++) csz *= g.cdims[i];
  for(int j = 0; j < lc.nk; j++) k *= t.adims[lc.k_a[j]];
  for(int j = 0; j < lc.nar; j++) k *= t.adims[lc.ar_a[j]];
  for(int j = 0; j < lc.nbr; j++) k *= t.bdims[lc.br_b[j]];
  return 2.0 * csz * k;
}

void finalize_worklist(const LabelClasses& lc, WorkList& wl, bool upload) {
  wl.flops_run = 0;
  for(const auto& g: wl.groups) {
    TB_EXPECTS(g.task_begin >= 0 && g.task_end >= g.task_begin &&
                 g.task_end <= (int64_t) wl.tasks.size(),
               "group task range out of bounds");
    for(int t = g.task_begin; t < g.task_end; t++) {
      validate_task(lc, g, wl.tasks[t]);
      wl.flops_run += task_flops(lc, g, wl.tasks[t]);
    }
  }
  wl.flops = wl.flops_run + wl.flops_skipped;
  if(!upload) return;
  TB_CUDA(cudaGetDevice(&wl.device));
  auto up = [](auto*& dptr, const auto& vec) {
    using T = std::remove_reference_t<decltype(vec[0])>;
    if(vec.empty()) return;
    TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&dptr), sizeof(T) * vec.size()));
    TB_CUDA(cudaMemcpy(dptr, vec.data(), sizeof(T) * vec.size(), cudaMemcpyHostToDevice));
  };
  up(wl.d_groups, wl.groups);
  up(wl.d_tasks, wl.tasks);
}

WorkList* single_block_worklist(const LabelClasses& lc, const int64_t* adims, const int64_t* bdims,
                                const int64_t* cdims) {
  auto*    wl = new WorkList();
  DevGroup g{};
  g.c_off      = 0;
  g.task_begin = 0;
  g.task_end   = 1;
  for(int i = 0; i < lc.nc; i++) {
    TB_EXPECTS(cdims[i] > 0 && cdims[i] < (1ll << 31), "block extent out of range");
    g.cdims[i] = (int32_t) cdims[i];
  }
  DevTask t{};
  for(int i = 0; i < lc.na; i++) {
    TB_EXPECTS(adims[i] > 0 && adims[i] < (1ll << 31), "block extent out of range");
    t.adims[i] = (int32_t) adims[i];
  }
  for(int i = 0; i < lc.nb; i++) {
    TB_EXPECTS(bdims[i] > 0 && bdims[i] < (1ll << 31), "block extent out of range");
    t.bdims[i] = (int32_t) bdims[i];
  }
  wl->groups.push_back(g);
  wl->tasks.push_back(t);
  return wl;
}

} // namespace tb
