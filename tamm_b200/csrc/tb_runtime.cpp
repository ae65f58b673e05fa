// Runtime tier implementation: arena, index spaces, tiling, block store, Scheduler.
#include "tb_runtime.hpp"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <numeric>
#include <sstream>

namespace tb {

uint64_t next_serial() {
  static std::atomic<uint64_t> n{0};
  return ++n;
}

// ------------------------------------------------------------------------- arena

Arena::Arena(int device, int64_t bytes): device_(device) {
  TB_EXPECTS(bytes > 0, "arena size must be positive");
  capacity_ = (bytes + 255) & ~int64_t(255);
  TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&base_), (size_t) capacity_));
  add_free(0, capacity_);
}

void Arena::add_free(int64_t off, int64_t size) {
  free_[off] = size;
  by_size_.insert({size, off});
}

void Arena::drop_free(std::map<int64_t, int64_t>::iterator it) {
  by_size_.erase({it->second, it->first});
  free_.erase(it);
}

Arena::~Arena() {
  if(base_) {
    int cur = -1;
    cudaGetDevice(&cur);
    cudaSetDevice(device_);
    cudaFree(base_);
    if(cur >= 0) cudaSetDevice(cur);
  }
}

void* Arena::allocate(int64_t bytes) {
  if(bytes <= 0) bytes = 1;
  const int64_t need = (bytes + 255) & ~int64_t(255);
  const auto    fit  = by_size_.lower_bound({need, int64_t(0)}); // best fit: smallest block that holds it
  if(fit == by_size_.end()) {
    std::ostringstream os;
    os << "device arena exhausted: need " << need << " bytes, " << (capacity_ - used_)
       << " free of " << capacity_ << " (fragmented)";
    fail(TB_ERR_NO_MEMORY, os.str());
  }
  const int64_t off = fit->second, sz = fit->first;
  drop_free(free_.find(off));
  if(sz > need) add_free(off + need, sz - need);
  inuse_[off] = need;
  used_ += need;
  peak_ = std::max(peak_, used_);
  return base_ + off;
}

void Arena::deallocate(void* p) {
  if(p == nullptr) return;
  const int64_t off = static_cast<char*>(p) - base_;
  auto          it  = inuse_.find(off);
  TB_EXPECTS(it != inuse_.end(), "pointer does not belong to this arena");
  int64_t sz = it->second;
  inuse_.erase(it);
  used_ -= sz;
  int64_t start = off;
  auto    nx    = free_.lower_bound(off); // coalesce with neighbours
  if(nx != free_.end() && nx->first == off + sz) {
    sz += nx->second;
    auto after = std::next(nx);
    drop_free(nx);
    nx = after;
  }
  if(nx != free_.begin()) {
    auto pv = std::prev(nx);
    if(pv->first + pv->second == start) {
      start = pv->first;
      sz += pv->second;
      drop_free(pv);
    }
  }
  add_free(start, sz);
}

void* Scratch::get(int64_t bytes) {
  if(arena) return arena->allocate(bytes);
  void* p = nullptr;
  TB_CUDA(cudaMallocAsync(&p, (size_t) std::max<int64_t>(bytes, 1), stream));
  return p;
}

void Scratch::put(void* p) {
  if(p == nullptr) return;
  if(arena) arena->deallocate(p);
  else TB_CUDA(cudaFreeAsync(p, stream));
}

void* CapturePool::get(int64_t bytes) {
  bytes = std::max<int64_t>(bytes, 1);
  int best = -1;
  for(int i = 0; i < (int) bufs.size(); i++)
    if(!std::get<2>(bufs[i]) && std::get<1>(bufs[i]) >= bytes &&
       (best < 0 || std::get<1>(bufs[i]) < std::get<1>(bufs[best])))
      best = i;
  if(best < 0) {
    bufs.emplace_back(arena->allocate(bytes), bytes, false);
    best = (int) bufs.size() - 1;
  }
  std::get<2>(bufs[best]) = true;
  return std::get<0>(bufs[best]);
}

void CapturePool::put(void* p) {
  for(auto& b: bufs)
    if(std::get<0>(b) == p) std::get<2>(b) = false;
}

void CapturePool::release() {
  for(auto& b: bufs) arena->deallocate(std::get<0>(b));
  bufs.clear();
}

Ctx::~Ctx() {
  if(stream) {
    cudaSetDevice(device);
    cudaStreamSynchronize(stream);
    for(cudaStream_t x: {h2d, d2h})
      if(x) {
        cudaStreamSynchronize(x);
        cudaStreamDestroy(x);
      }
    arena.reset();
    cudaStreamDestroy(stream);
  }
}

Tensor::~Tensor() {
  if(used || filled) {
    if(ctx) cudaSetDevice(ctx->device);
    if(used) cudaEventDestroy(used);
    if(filled) cudaEventDestroy(filled);
  }
}

// marks the end of the compute work enqueued so far that touched t
static void mark_used(Tensor* t, cudaStream_t st) {
  if(!t || !t->data) return;
  if(!t->used) TB_CUDA(cudaEventCreateWithFlags(&t->used, cudaEventDisableTiming));
  TB_CUDA(cudaEventRecord(t->used, st));
}

// ------------------------------------------------------------------ index spaces

int IndexSpace::spin_of(int64_t idx) const {
  for(const auto& kv: spin)
    for(const auto& r: kv.second)
      if(idx >= r.first && idx < r.second) return kv.first;
  return 0; // default spin of an unattributed index (index_space_interface.hpp:466-468)
}

std::vector<int64_t> IndexSpace::boundaries(bool with_named) const {
  std::vector<int64_t> b;
  if(with_named)
    for(const auto& kv: named)
      for(const auto& r: kv.second) {
        b.push_back(r.first);
        b.push_back(r.second);
      }
  for(const auto& kv: spin)
    for(const auto& r: kv.second) {
      b.push_back(r.first);
      b.push_back(r.second);
    }
  std::sort(b.begin(), b.end());
  b.erase(std::unique(b.begin(), b.end()), b.end());
  return b;
}

int64_t TIS::find_root(int64_t r) const {
  auto it = std::find(tiles.begin(), tiles.end(), r);
  return it == tiles.end() ? -1 : (int64_t) (it - tiles.begin());
}

// TiledIndexSpaceInfo::construct_tiled_indices (tiled_index_space.hpp:1135-1194 for a
// uniform tile size, :1205-1262 for a tile list).
std::shared_ptr<TIS> make_tis(const std::shared_ptr<IndexSpace>& is, int64_t tile,
                              const int64_t* tiles, int64_t ntiles) {
  auto root = std::make_shared<RootTiling>();
  root->is  = is;
  auto& off = root->offsets;
  if(is->n == 0) off.push_back(0);
  else if(tiles == nullptr) {
    TB_EXPECTS(tile > 0, "tile size must be positive");
    auto b = is->boundaries(true);
    if(b.empty()) {
      for(int64_t i = 0; i < is->n; i += tile) off.push_back(i);
    }
    else {
      int64_t i = 0;
      size_t  j = (i == b[0]) ? 1 : 0;
      while(i < is->n) {
        off.push_back(i);
        if(j < b.size() && i + tile >= b[j]) i = b[j++];
        else i = i + tile;
      }
    }
    off.push_back(is->n);
  }
  else {
    int64_t sum = 0;
    for(int64_t t = 0; t < ntiles; t++) {
      TB_EXPECTS(tiles[t] > 0, "tile sizes must be positive");
      sum += tiles[t];
    }
    TB_EXPECTS(sum == is->n, "tile sizes do not add up to the index space size");
    int64_t j = 0;
    for(int64_t i = 0; i < is->n; i += tiles[j++]) off.push_back(i);
    off.push_back(is->n);
    for(int64_t bnd: is->boundaries(true))
      TB_EXPECTS(std::binary_search(off.begin(), off.end(), bnd),
                 "tile list does not split at every named/spin boundary");
  }
  const int64_t nt = (int64_t) off.size() - 1;
  root->spins.resize(nt > 0 ? nt : 0);
  for(int64_t t = 0; t < nt; t++) root->spins[t] = is->spin_of(off[t]);
  auto s  = std::make_shared<TIS>();
  s->root = root;
  s->tiles.resize(nt > 0 ? nt : 0);
  std::iota(s->tiles.begin(), s->tiles.end(), 0);
  return s;
}

std::shared_ptr<TIS> tis_named(const TIS& parent, const std::string& name) {
  const auto& is = *parent.root->is;
  const std::vector<Range>* ranges = nullptr;
  for(const auto& kv: is.named)
    if(kv.first == name) ranges = &kv.second;
  if(name == "all") {
    auto s   = std::make_shared<TIS>(parent);
    return s;
  }
  TB_EXPECTS(ranges != nullptr, "no named subspace '" + name + "'");
  auto s  = std::make_shared<TIS>();
  s->root = parent.root;
  for(int64_t t: parent.tiles) {
    const int64_t lo = parent.root->offsets[t];
    for(const auto& r: *ranges)
      if(lo >= r.first && lo < r.second) {
        s->tiles.push_back(t);
        break;
      }
  }
  return s;
}

std::shared_ptr<TIS> tis_subrange(const TIS& parent, int64_t first, int64_t last) {
  TB_EXPECTS(first >= 0 && last >= first && last <= parent.ntiles(), "tile range out of bounds");
  TB_EXPECTS(!parent.dep, "tile sub-ranges of a dependent space are not supported");
  auto s  = std::make_shared<TIS>();
  s->root = parent.root;
  s->tiles.assign(parent.tiles.begin() + first, parent.tiles.begin() + last);
  return s;
}

// ---------------------------------------------------------------------- tensors

void Tensor::build_table() {
  key_stride.assign(nmodes, 1);
  for(int i = nmodes - 2; i >= 0; i--) key_stride[i] = key_stride[i + 1] * tis[i + 1]->ntiles();
  keys.clear();
  offsets.clear();
  std::vector<std::pair<int64_t, int64_t>> h;
  int64_t                                  nall = 1;
  for(int i = 0; i < nmodes; i++) nall *= tis[i]->ntiles();
  std::vector<int64_t> id(nmodes, 0);
  for(int64_t lin = 0; lin < nall; lin++) {
    if(is_non_zero(id.data())) h.push_back({key(id.data()), block_size(id.data())});
    for(int q = nmodes - 1; q >= 0; q--) {
      if(++id[q] < tis[q]->ntiles()) break;
      id[q] = 0;
    }
  }
  std::sort(h.begin(), h.end());
  int64_t off = 0;
  for(const auto& kv: h) {
    keys.push_back(kv.first);
    offsets.push_back(off);
    off += kv.second;
  }
  nelems = off;
}

bool Tensor::is_non_zero(const int64_t* blockid) const {
  // dependent modes: the block exists only where the tile of the dependent mode is one
  // of the tiles its space lists for the tiles of the modes it depends on
  // (translate_blockid_if_possible, utils.hpp:369)
  for(int m = 0; m < (int) dep_modes.size(); m++) {
    if(dep_modes[m].empty()) continue;
    const Dependency&    d = *tis[m]->dep;
    std::vector<int64_t> key(dep_modes[m].size());
    for(size_t k = 0; k < key.size(); k++) {
      const int o = dep_modes[m][k];
      key[k]      = d.on[k]->find_root(tis[o]->tiles[blockid[o]]);
      if(key[k] < 0) return false;
    }
    auto it = d.valid.find(key);
    if(it == d.valid.end() || !it->second[blockid[m]]) return false;
  }
  // TensorBase::is_non_zero (tensor_base.hpp:243-263)
  if(!has_spin) return true;
  int upper = 0, lower = 0;
  for(int i = 0; i < nmodes; i++) {
    if(mask[i] == 0) upper += tis[i]->spin(blockid[i]);
    else if(mask[i] == 1) lower += tis[i]->spin(blockid[i]);
  }
  return upper == lower;
}

int64_t Tensor::key(const int64_t* blockid) const {
  int64_t k = 0;
  for(int i = 0; i < nmodes; i++) k += blockid[i] * key_stride[i];
  return k;
}

int64_t Tensor::locate(const int64_t* blockid) const {
  const int64_t k  = key(blockid);
  auto          it = std::lower_bound(keys.begin(), keys.end(), k);
  if(it == keys.end() || *it != k) return -1;
  return offsets[it - keys.begin()];
}

int64_t Tensor::block_size(const int64_t* blockid) const {
  int64_t s = 1;
  for(int i = 0; i < nmodes; i++) s *= tis[i]->size(blockid[i]);
  return s;
}

void Tensor::block_dims(const int64_t* blockid, int32_t* dims) const {
  for(int i = 0; i < nmodes; i++) dims[i] = (int32_t) tis[i]->size(blockid[i]);
}

void Tensor::check_blockid(const int64_t* blockid) const {
  for(int i = 0; i < nmodes; i++)
    TB_EXPECTS(blockid[i] >= 0 && blockid[i] < tis[i]->ntiles(), "block id out of range");
}

void Tensor::require_allocated() const {
  if(is_lambda() && data == nullptr)
    fail(TB_ERR_NOT_IMPLEMENTED, "a lambda tensor can only be read by a contraction (its blocks exist on demand)");
  if(data == nullptr && nelems > 0) fail(TB_ERR_STATE, "tensor is not allocated");
}

void Tensor::require_writable() const {
  if(read_only) fail(TB_ERR_STATE, "tensor is marked read-only (tb_tensor_set_read_only)");
}

int64_t Tensor::block_index(const int64_t* blockid) const {
  const int64_t k  = key(blockid);
  auto          it = std::lower_bound(keys.begin(), keys.end(), k);
  return (it != keys.end() && *it == k) ? (int64_t) (it - keys.begin()) : -1;
}

bool Tensor::block_is_zero(const int64_t* blockid) const {
  if(!read_only) return false;
  const int64_t k  = key(blockid);
  auto          it = std::lower_bound(keys.begin(), keys.end(), k);
  return it != keys.end() && *it == k && zero_block[it - keys.begin()] != 0;
}

// Sets or clears the read-only mark.  Setting it scans the stored blocks once on the
// context's stream (after the work already enqueued there, which includes the waits
// for asynchronous host writes) for blocks whose elements are all zero.
void set_read_only(Tensor& T, bool on) {
  for(auto& kv: T.digit_cache) kv.second->retire(); // memory back now, even if a layout refers to it
  T.digit_cache.clear();
  if(!on) {
    T.read_only = false;
    T.zero_block.clear();
    return;
  }
  T.require_allocated();
  const int64_t nb = (int64_t) T.keys.size();
  TB_EXPECTS(nb < (1ll << 31), "too many blocks");
  std::vector<int64_t>  pairs(2 * std::max<int64_t>(nb, 1));
  std::vector<uint32_t> nz(std::max<int64_t>(nb, 1), 1u);
  for(int64_t b = 0; b < nb; b++) {
    pairs[2 * b]     = T.offsets[b];
    pairs[2 * b + 1] = (b + 1 < nb ? T.offsets[b + 1] : T.nelems) - T.offsets[b];
  }
  if(nb > 0) {
    Ctx& c = *T.ctx;
    TB_CUDA(cudaSetDevice(c.device));
    auto* dp = static_cast<int64_t*>(c.arena->allocate((int64_t) sizeof(int64_t) * 2 * nb));
    auto* dn = static_cast<uint32_t*>(c.arena->allocate((int64_t) sizeof(uint32_t) * nb));
    TB_CUDA(cudaMemcpyAsync(dp, pairs.data(), sizeof(int64_t) * 2 * nb, cudaMemcpyHostToDevice, c.stream));
    launch_block_nonzero(T.data, dp, (int) nb, dn, c.stream);
    TB_CUDA(cudaMemcpyAsync(nz.data(), dn, sizeof(uint32_t) * nb, cudaMemcpyDeviceToHost, c.stream));
    TB_CUDA(cudaStreamSynchronize(c.stream));
    c.arena->deallocate(dn);
    c.arena->deallocate(dp);
  }
  T.zero_block.assign(nb, 0);
  for(int64_t b = 0; b < nb; b++) T.zero_block[b] = nz[b] ? 0 : 1;
  T.read_only = true;
  T.ro_serial = next_serial();
}

// -------------------------------------------------------------------- scheduler

namespace {

int find_label(const std::vector<int>& v, int x) {
  for(size_t i = 0; i < v.size(); i++)
    if(v[i] == x) return (int) i;
  return -1;
}

// label-space tile -> tensor tile for every mode (internal::translate_blockid,
// utils.hpp:264-286), -1 where the label tile is not a tile of the tensor's space
std::vector<std::vector<int64_t>> tile_maps(const Labeled& x) {
  std::vector<std::vector<int64_t>> m(x.t->nmodes);
  for(int i = 0; i < x.t->nmodes; i++) {
    const TIS& ls = *x.ltis[i];
    const TIS& ts = *x.t->tis[i];
    TB_EXPECTS(ls.root == ts.root, "label space and tensor space do not share a root tiling");
    m[i].resize(ls.ntiles());
    for(int64_t t = 0; t < ls.ntiles(); t++) {
      m[i][t] = ts.find_root(ls.tiles[t]);
      TB_EXPECTS(m[i][t] >= 0, "label tile is not a tile of the tensor's index space");
    }
  }
  return m;
}

bool next_tuple(std::vector<int64_t>& it, const std::vector<int64_t>& nt) {
  for(int q = (int) it.size() - 1; q >= 0; q--) {
    if(++it[q] < nt[q]) return true;
    it[q] = 0;
  }
  return false;
}

// Same tensor, labels and label spaces.
bool same_target(const Labeled& x, const Labeled& y) {
  if(x.t != y.t || x.labels != y.labels || x.ltis.size() != y.ltis.size()) return false;
  for(size_t i = 0; i < x.ltis.size(); i++)
    if(x.ltis[i].get() != y.ltis[i].get()) return false;
  return true;
}

std::string signature(const Op& op) {
  std::ostringstream os;
  auto               put = [&](const Labeled& x) {
    os << x.t << "#" << x.t->serial.v << "r" << (x.t->read_only ? x.t->ro_serial : 0) << ":";
    for(size_t i = 0; i < x.labels.size(); i++)
      os << x.labels[i] << "@" << x.ltis[i].get() << "#" << x.ltis[i]->serial.v << ",";
    os << "|";
  };
  os << (int) op.kind << "|";
  if(op.kind == Op::Map) os << "f" << op.fn << "|";
  put(op.lhs);
  if(op.kind != Op::Set) put(op.a);
  if(op.kind == Op::Mult) put(op.b);
  return os.str();
}

// MultOp::execute_bufacc enumeration (multop.hpp:576-893): owned admitted output
// blocks x admitted reduction tiles, as device work-list groups and tasks.
// Owner of each output block for nranks processes: blocks in decreasing FP64 work
// (ties by position), each to the rank with the least work so far (ties to the lower
// rank).  Every rank computes the same assignment from the same work list, so no
// exchange is needed to agree on it (the role of TAMM's owner-computes rule,
// multop.hpp:880-891, with a FLOP-balanced distribution instead of GA's).
std::vector<int> group_owners(const LabelClasses& lc, const WorkList& wl, int nranks) {
  std::vector<double> work(wl.groups.size(), 0.0);
  for(size_t g = 0; g < wl.groups.size(); g++)
    for(int t = wl.groups[g].task_begin; t < wl.groups[g].task_end; t++)
      work[g] += task_flops(lc, wl.groups[g], wl.tasks[t]);
  std::vector<size_t> order(wl.groups.size());
  for(size_t g = 0; g < order.size(); g++) order[g] = g;
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return work[x] > work[y]; });
  std::vector<double> load(nranks, 0.0);
  std::vector<int>    owner(wl.groups.size(), 0);
  for(size_t g: order) {
    int r = 0;
    for(int q = 1; q < nranks; q++)
      if(load[q] < load[r]) r = q;
    owner[g] = r;
    load[r] += work[g];
  }
  return owner;
}

std::shared_ptr<WorkList> build_mult_worklist(const Op& op, const LabelClasses& lc, bool upload, int rank,
                                              int nranks) {
  const Labeled &c = op.lhs, &a = op.a, &b = op.b;
  auto cm = tile_maps(c), am = tile_maps(a), bm = tile_maps(b);
  // reduction labels: unique rhs labels (A then B) not in the lhs, sorted (multop.hpp:593-601)
  std::vector<int>                 red;
  std::map<int, const TIS*>        lsp;
  auto note = [&](const Labeled& x) {
    for(size_t i = 0; i < x.labels.size(); i++) {
      auto it = lsp.find(x.labels[i]);
      if(it == lsp.end()) lsp[x.labels[i]] = x.ltis[i].get();
      else
        TB_EXPECTS(it->second->root == x.ltis[i]->root && it->second->tiles == x.ltis[i]->tiles,
                   "one label bound to two different index spaces");
    }
  };
  note(c);
  note(a);
  note(b);
  for(int l: a.labels)
    if(find_label(c.labels, l) < 0 && find_label(red, l) < 0) red.push_back(l);
  for(int l: b.labels)
    if(find_label(c.labels, l) < 0 && find_label(red, l) < 0) red.push_back(l);
  std::sort(red.begin(), red.end());
  std::vector<int64_t> red_nt, c_nt;
  for(int l: red) red_nt.push_back(lsp[l]->ntiles());
  for(size_t i = 0; i < c.labels.size(); i++) c_nt.push_back(c.ltis[i]->ntiles());
  std::vector<int> a_out(a.labels.size()), a_red(a.labels.size()), b_out(b.labels.size()),
    b_red(b.labels.size());
  for(size_t i = 0; i < a.labels.size(); i++) {
    a_out[i] = find_label(c.labels, a.labels[i]);
    a_red[i] = find_label(red, a.labels[i]);
  }
  for(size_t i = 0; i < b.labels.size(); i++) {
    b_out[i] = find_label(c.labels, b.labels[i]);
    b_red[i] = find_label(red, b.labels[i]);
  }

  auto wl = std::make_shared<WorkList>();
  for(int64_t n: c_nt)
    if(n == 0) return wl;
  for(int64_t n: red_nt)
    if(n == 0) return wl;
  std::vector<int64_t> itval(c.labels.size(), 0), inner(red.size(), 0);
  std::vector<int64_t> cid(c.labels.size()), aid(a.labels.size()), bid(b.labels.size());
  std::vector<double>  skip_flops; // per group
  std::vector<int64_t> skip_count;
  do {
    for(size_t i = 0; i < cid.size(); i++) cid[i] = cm[i][itval[i]];
    if(!c.t->is_non_zero(cid.data())) continue;
    DevGroup g{};
    g.c_off = c.t->locate(cid.data());
    c.t->block_dims(cid.data(), g.cdims);
    g.task_begin = (int32_t) wl->tasks.size();
    std::fill(inner.begin(), inner.end(), 0);
    double  gskip  = 0; // FLOPs and count of this group's skipped tasks
    int64_t gskipn = 0;
    do {
      for(size_t i = 0; i < aid.size(); i++) {
        int64_t l = a_out[i] >= 0 ? itval[a_out[i]] : inner[a_red[i]];
        aid[i]    = am[i][l];
      }
      if(!a.t->is_non_zero(aid.data())) continue;
      for(size_t i = 0; i < bid.size(); i++) {
        int64_t l = b_out[i] >= 0 ? itval[b_out[i]] : inner[b_red[i]];
        bid[i]    = bm[i][l];
      }
      if(!b.t->is_non_zero(bid.data())) continue;
      DevTask t{};
      t.a_off = a.t->locate(aid.data());
      t.b_off = b.t->locate(bid.data());
      a.t->block_dims(aid.data(), t.adims);
      b.t->block_dims(bid.data(), t.bdims);
      // an admitted task over an exactly-zero block of a read-only operand, or over a
      // block that an earlier assignment of the same op list left without any
      // contribution, adds exactly zero to C: it is counted, not run
      if(a.t->block_is_zero(aid.data()) || b.t->block_is_zero(bid.data()) ||
         (op.za && (*op.za)[a.t->block_index(aid.data())]) || (op.zb && (*op.zb)[b.t->block_index(bid.data())])) {
        gskip += task_flops(lc, g, t);
        gskipn++;
        continue;
      }
      wl->tasks.push_back(t);
    } while(!red.empty() && next_tuple(inner, red_nt));
    TB_EXPECTS(wl->tasks.size() < (1ull << 31), "too many tasks in one contraction");
    g.task_end = (int32_t) wl->tasks.size();
    wl->groups.push_back(g);
    skip_flops.push_back(gskip);
    skip_count.push_back(gskipn);
  } while(!cid.empty() && next_tuple(itval, c_nt));
  if(nranks > 1) { // keep the output blocks this rank owns
    const std::vector<int> owner = group_owners(lc, *wl, nranks);
    auto                   mine  = std::make_shared<WorkList>();
    for(size_t gi = 0; gi < wl->groups.size(); gi++) {
      if(owner[gi] != rank) continue;
      mine->flops_skipped += skip_flops[gi];
      mine->ntasks_skipped += skip_count[gi];
      DevGroup g   = wl->groups[gi];
      g.task_begin = (int32_t) mine->tasks.size();
      for(int t = wl->groups[gi].task_begin; t < wl->groups[gi].task_end; t++) mine->tasks.push_back(wl->tasks[t]);
      g.task_end = (int32_t) mine->tasks.size();
      mine->groups.push_back(g);
    }
    wl = mine;
  }
  else
    for(size_t gi = 0; gi < wl->groups.size(); gi++) {
      wl->flops_skipped += skip_flops[gi];
      wl->ntasks_skipped += skip_count[gi];
    }
  finalize_worklist(lc, *wl, upload);
  return wl;
}

} // namespace

std::shared_ptr<WorkList> mult_worklist(const Op& op, const LabelClasses& lc, bool upload, int rank, int nranks) {
  return build_mult_worklist(op, lc, upload, rank, nranks);
}

void run_contract(Plan& plan, const WorkList& wl, double alpha, const double* A, const double* B,
                  double* C, cudaStream_t stream, Arena* arena); // tb_capi.cpp
static std::shared_ptr<EnergySpec> build_energy(const Op& op, const LabelClasses& lc, const std::shared_ptr<Ctx>& ctx);

void Sched::run(Op& op) {
  cudaStream_t st = ctx->stream;
  if(op.kind == Op::Set || op.kind == Op::Add || (op.kind == Op::Mult && !op.energy) || op.kind == Op::Denom ||
     op.kind == Op::Map)
    op.lhs.t->require_writable();
  if(op.kind == Op::Map) {
    op.lhs.t->require_allocated();
    op.a.t->require_allocated();
    if(!op.map_dev) {
      const std::string key = "M|" + signature(op);
      auto&             cached = fill_cache[key];
      auto&             count  = map_count[key];
      if(!cached) {
        // MapOp's loop over the lhs label tuples (mapop.hpp:52-90): every admitted lhs
        // block, the rhs block with the same label tiles (or zeros where not stored)
        auto                 lm = tile_maps(op.lhs), rm = tile_maps(op.a);
        std::vector<int64_t> nt, it(op.lhs.t->nmodes, 0), lid(op.lhs.t->nmodes), rid(op.a.t->nmodes), tri;
        for(int i = 0; i < op.lhs.t->nmodes; i++) nt.push_back(op.lhs.ltis[i]->ntiles());
        bool empty = false;
        for(auto n: nt) empty |= (n == 0);
        if(!empty) do {
            for(int i = 0; i < op.lhs.t->nmodes; i++) {
              lid[i] = lm[i][it[i]];
              rid[i] = rm[i][it[i]];
            }
            if(!op.lhs.t->is_non_zero(lid.data())) continue;
            const int64_t n = op.lhs.t->block_size(lid.data());
            TB_EXPECTS(op.a.t->block_size(rid.data()) == n, "map: lhs and rhs blocks differ in size");
            tri.push_back(op.lhs.t->locate(lid.data()));
            tri.push_back(op.a.t->is_non_zero(rid.data()) ? op.a.t->locate(rid.data()) : -1);
            tri.push_back(n);
          } while(!it.empty() && next_tuple(it, nt));
        TB_EXPECTS(tri.size() / 3 < (1u << 31), "too many blocks in one map");
        const std::vector<int64_t> segs = seg_list(tri);
        int64_t*                   d    = nullptr;
        const int                  dev  = ctx->device;
        TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&d), sizeof(int64_t) * std::max<size_t>(segs.size(), 1)));
        cached = std::shared_ptr<int64_t>(d, [dev](int64_t* q) {
          int cur = -1;
          cudaGetDevice(&cur);
          cudaSetDevice(dev);
          cudaFree(q);
          if(cur >= 0) cudaSetDevice(cur);
        });
        if(!segs.empty())
          TB_CUDA(cudaMemcpy(d, segs.data(), sizeof(int64_t) * segs.size(), cudaMemcpyHostToDevice));
        count           = (int) (segs.size() / 4);
        seg_total[key]  = segs.empty() ? 0 : segs[segs.size() - 1] + segs[segs.size() - 2];
      }
      op.map_dev   = cached;
      op.map_n     = count;
      op.map_total = seg_total[key];
    }
    launch_map_blocks(op.lhs.t->data, op.a.t->data, op.map_dev.get(), op.map_n, op.map_total, op.fn, op.value, st);
    return;
  }
  if(op.kind == Op::Set) {
    op.lhs.t->require_allocated();
    if(op.fill_none) return;
    if(!op.set_blocks) {
      auto blocks = std::make_shared<std::vector<int64_t>>();
      bool whole  = true;
      for(int i = 0; i < op.lhs.t->nmodes; i++)
        if(op.lhs.ltis[i]->tiles != op.lhs.t->tis[i]->tiles) whole = false;
      if(!whole) {
        auto                 m = tile_maps(op.lhs);
        std::vector<int64_t> nt, it(op.lhs.t->nmodes, 0), id(op.lhs.t->nmodes);
        for(int i = 0; i < op.lhs.t->nmodes; i++) nt.push_back(op.lhs.ltis[i]->ntiles());
        bool empty = false;
        for(auto n: nt) empty |= (n == 0);
        if(!empty) do {
            for(int i = 0; i < op.lhs.t->nmodes; i++) id[i] = m[i][it[i]];
            if(!op.lhs.t->is_non_zero(id.data())) continue;
            blocks->push_back(op.lhs.t->locate(id.data()));
            blocks->push_back(op.lhs.t->block_size(id.data()));
          } while(!it.empty() && next_tuple(it, nt));
      }
      op.set_blocks = blocks;
    }
    if(op.set_blocks->empty()) launch_fill(op.lhs.t->data, op.lhs.t->nelems, op.value, op.is_assign, st);
    else {
      const size_t nb = op.set_blocks->size() / 2;
      TB_EXPECTS(nb < (1u << 31), "too many blocks in one fill");
      if(!op.set_dev) { // one upload per signature; later ops and graph replays reuse it
        if(op.fill_key.empty()) op.fill_key = "S|" + signature(op);
        auto& cached = fill_cache[op.fill_key];
        if(!cached) {
          std::vector<int64_t> tri;
          for(size_t i = 0; i < nb; i++) {
            tri.push_back((*op.set_blocks)[2 * i]);
            tri.push_back(-1);
            tri.push_back((*op.set_blocks)[2 * i + 1]);
          }
          const std::vector<int64_t> segs = seg_list(tri);
          int64_t*                   d    = nullptr;
          const int                  dev  = ctx->device;
          TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&d), sizeof(int64_t) * std::max<size_t>(segs.size(), 1)));
          cached = std::shared_ptr<int64_t>(d, [dev](int64_t* p) {
            int cur = -1;
            cudaGetDevice(&cur);
            cudaSetDevice(dev);
            cudaFree(p);
            if(cur >= 0) cudaSetDevice(cur);
          });
          if(!segs.empty())
            TB_CUDA(cudaMemcpy(d, segs.data(), sizeof(int64_t) * segs.size(), cudaMemcpyHostToDevice));
          map_count[op.fill_key] = (int) (segs.size() / 4);
          seg_total[op.fill_key] = segs.empty() ? 0 : segs[segs.size() - 1] + segs[segs.size() - 2];
        }
        op.set_dev   = cached;
        op.set_nseg  = map_count[op.fill_key];
        op.set_total = seg_total[op.fill_key];
      }
      launch_fill_blocks(op.lhs.t->data, op.set_dev.get(), op.set_nseg, op.set_total, op.value, op.is_assign, st);
    }
    return;
  }
  if(op.kind == Op::Add) {
    op.lhs.t->require_allocated();
    op.a.t->require_allocated();
    if(!op.add_blocks) {
      auto blocks = std::make_shared<std::vector<Op::AddBlock>>();
      // FlatAddPlan condition (addop.hpp:245-251): same labels, same layout
      bool flat = op.lhs.labels == op.a.labels && op.lhs.t->has_spin == op.a.t->has_spin &&
                  op.lhs.t->nmodes == op.a.t->nmodes && op.lhs.t->keys == op.a.t->keys &&
                  op.lhs.t->offsets == op.a.t->offsets;
      for(int i = 0; flat && i < op.lhs.t->nmodes; i++)
        flat = op.lhs.ltis[i]->tiles == op.lhs.t->tis[i]->tiles &&
               op.a.ltis[i]->tiles == op.a.t->tis[i]->tiles &&
               op.lhs.t->tis[i]->tiles == op.a.t->tis[i]->tiles &&
               op.lhs.t->tis[i]->root == op.a.t->tis[i]->root;
      op.flat = flat;
      if(!flat) {
        // LHSAddPlan (addop.hpp:457-519): loop over the merged labels, skip pairs with
        // a non-admitted side, apply the block assign.
        auto             lm = tile_maps(op.lhs), rm = tile_maps(op.a);
        std::vector<int> merged = op.lhs.labels;
        std::vector<const TIS*> msp;
        for(size_t i = 0; i < op.lhs.labels.size(); i++) msp.push_back(op.lhs.ltis[i].get());
        for(size_t i = 0; i < op.a.labels.size(); i++)
          if(find_label(merged, op.a.labels[i]) < 0) {
            merged.push_back(op.a.labels[i]);
            msp.push_back(op.a.ltis[i].get());
          }
        std::vector<int64_t> nt, it(merged.size(), 0);
        for(auto* s: msp) nt.push_back(s->ntiles());
        bool empty = false;
        for(auto n: nt) empty |= (n == 0);
        std::vector<int64_t> lid(op.lhs.t->nmodes), rid(op.a.t->nmodes);
        if(!empty) do {
            for(int i = 0; i < op.lhs.t->nmodes; i++) lid[i] = lm[i][it[find_label(merged, op.lhs.labels[i])]];
            for(int i = 0; i < op.a.t->nmodes; i++) rid[i] = rm[i][it[find_label(merged, op.a.labels[i])]];
            if(!op.lhs.t->is_non_zero(lid.data()) || !op.a.t->is_non_zero(rid.data())) continue;
            Op::AddBlock ab{};
            ab.dst_off = op.lhs.t->locate(lid.data());
            ab.src_off = op.a.t->locate(rid.data());
            for(int i = 0; i < op.lhs.t->nmodes; i++) ab.ddims[i] = op.lhs.t->tis[i]->size(lid[i]);
            for(int i = 0; i < op.a.t->nmodes; i++) ab.sdims[i] = op.a.t->tis[i]->size(rid[i]);
            blocks->push_back(ab);
          } while(!it.empty() && next_tuple(it, nt));
      }
      op.add_blocks = blocks;
    }
    if(op.flat) {
      launch_axpby(op.alpha, op.a.t->data, op.is_assign ? 0.0 : 1.0, op.lhs.t->data,
                   op.lhs.t->nelems, st);
      return;
    }
    if(!op.add_dev) { // every block pair in one launch; the list is uploaded once per signature
      const std::string key    = "A|" + signature(op);
      auto&             cached = fill_cache[key];
      auto&             count  = map_count[key];
      if(!cached) {
        std::vector<BlockAssign> list;
        int64_t                  units = 0;
        for(const auto& ab: *op.add_blocks) {
          AssignLoop lp = plan_assign(ab.ddims, op.lhs.labels.data(), op.lhs.t->nmodes, ab.sdims,
                                      op.a.labels.data(), op.a.t->nmodes);
          list.push_back(make_block_assign(lp, ab.dst_off, ab.src_off, units));
          units += list.back().units;
        }
        add_units[key] = units;
        TB_EXPECTS(list.size() < (1u << 31), "too many block pairs in one add");
        BlockAssign* d   = nullptr;
        const int    dev = ctx->device;
        TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&d), sizeof(BlockAssign) * std::max<size_t>(list.size(), 1)));
        cached = std::shared_ptr<int64_t>(reinterpret_cast<int64_t*>(d), [dev](int64_t* q) {
          int cur = -1;
          cudaGetDevice(&cur);
          cudaSetDevice(dev);
          cudaFree(q);
          if(cur >= 0) cudaSetDevice(cur);
        });
        if(!list.empty())
          TB_CUDA(cudaMemcpy(d, list.data(), sizeof(BlockAssign) * list.size(), cudaMemcpyHostToDevice));
        count = (int) list.size();
      }
      op.add_dev   = cached;
      op.add_n     = count;
      op.add_units = add_units[key];
    }
    launch_assign_blocks(op.lhs.t->data, op.alpha, op.a.t->data, reinterpret_cast<const BlockAssign*>(op.add_dev.get()),
                         op.add_n, op.add_units, op.is_assign, st);
    return;
  }
  if(op.kind == Op::Dot) {
    op.a.t->require_allocated();
    op.b.t->require_allocated();
    TB_EXPECTS(op.slot >= 0 && op.slot < kSlots, "scalar slot out of range (0..63)");
    launch_dot_to(op.a.t->data, op.root ? nullptr : op.b.t->data, op.a.t->nelems, op.alpha, op.root,
                  scalars() + op.slot, scalars() + kSlots, st);
    return;
  }
  if(op.kind == Op::Denom) {
    op.lhs.t->require_allocated();
    op.a.t->require_allocated();
    DenomSpec& d = *op.denom;
    if(!d.d_blocks) d.build(*op.lhs.t, ctx);
    DenomSigns sg{};
    for(int m = 0; m < kMaxModes; m++) sg.s[m] = d.signs[m];
    launch_denom(op.lhs.t->data, op.a.t->data, op.alpha, d.d_blocks, d.d_units, d.nunits, op.lhs.t->nmodes, d.d_eps,
                 sg, st);
    return;
  }
  if(op.kind == Op::DenomEnergy) {
    op.lhs.t->require_allocated();
    DenomSpec& d = *op.denom;
    if(!d.d_blocks) d.build(*op.lhs.t, ctx);
    DenomSigns sg{};
    for(int m = 0; m < kMaxModes; m++) sg.s[m] = d.signs[m];
    launch_denom_energy(op.lhs.t->data, op.alpha, d.d_blocks, d.d_units, d.nunits, op.lhs.t->nmodes, d.d_eps, sg,
                        d.d_part, scalars() + op.slot, st);
    return;
  }
  if(op.kind == Op::SetScalar) {
    launch_set_scalar(scalars() + op.slot, op.value, st);
    return;
  }
  // MultOp
  if(op.a.t->is_lambda() || op.b.t->is_lambda()) {
    if(op.energy) fail(TB_ERR_NOT_IMPLEMENTED, "energy epilogue with a lambda operand");
    run_lambda_mult(op);
    return;
  }
  op.lhs.t->require_allocated();
  op.a.t->require_allocated();
  op.b.t->require_allocated();
  prepare_mult(op);
  op.plan->mode       = ctx->mode;
  op.plan->err_target = ctx->err_target;
  op.plan->nslices    = ctx->nslices;
  op.plan->tile_n     = 0;
  op.plan->store      = op.store;
  op.plan->energy     = nullptr; // (plans are shared by signature: nothing of an earlier op stays)
  if(op.energy) { // the energy epilogue keeps the context's precision (no autotuning)
    if(!op.espec) op.espec = build_energy(op, op.plan->lc, ctx);
    op.plan->energy       = &op.espec->args;
    op.plan->energy_out   = scalars() + op.slot;
    op.plan->energy_scale = op.value;
  }
  else if(autotune && ctx->mode == TB_MODE_INT8 && !pinned) {
    const std::string key = signature(op) + "|" + std::to_string(ctx->err_target) + "|" + std::to_string(ctx->nslices);
    auto              it  = tune_cache.find(key);
    if(it == tune_cache.end()) {
      tune(op, key);
      it = tune_cache.find(key);
    }
    op.plan->mode   = it->second.mode;
    op.plan->tile_n = it->second.tile_n;
    op.tune_key     = key;
  }
  else if(autotune && ctx->mode == TB_MODE_INT8) { // capturing: the warm-up run tuned already
    auto it = tune_cache.find(signature(op) + "|" + std::to_string(ctx->err_target) + "|" +
                              std::to_string(ctx->nslices));
    if(it != tune_cache.end()) {
      op.plan->mode   = it->second.mode;
      op.plan->tile_n = it->second.tile_n;
    }
  }
  op.plan->profile      = profiling;
  op.plan->pinned       = pinned;
  op.plan->check_errors = pinned == nullptr && !deferred_checks;
  op.plan->cache_limit  = ctx->digit_cache_bytes;
  op.plan->cache_used   = &ctx->digit_cache_used;
  op.plan->cache_a      = ctx->digit_cache_bytes > 0 && op.a.t->read_only ? op.a.t : nullptr;
  op.plan->cache_b      = ctx->digit_cache_bytes > 0 && op.b.t->read_only ? op.b.t : nullptr;
  op.flops              = op.wl->flops;
  run_contract(*op.plan, *op.wl, op.alpha, op.a.t->data, op.b.t->data, op.lhs.t->data, st,
               ctx->arena.get());
  if(op.energy) {
    op.plan->energy = nullptr;
    if(const auto& r = op.espec->rest; r && r->nunits > 0) { // blocks of groups without tasks: C as it is
      DenomSigns sg{};
      for(int m = 0; m < kMaxModes; m++) sg.s[m] = r->signs[m];
      launch_denom_energy(op.lhs.t->data, op.value, r->d_blocks, r->d_units, r->nunits, op.lhs.t->nmodes, r->d_eps,
                          sg, r->d_part, scalars() + op.slot, st);
    }
  }
  op.plan->profile      = false;
  op.plan->pinned       = nullptr;
  op.plan->check_errors = true;
  op.plan->store        = false;
}

// Plan and work list of a MultOp, from the caches (keyed by the op's signature and
// this rank's share).
// Key of a structural-zero pattern: count of zero blocks and an FNV-1a hash of the bytes.
static std::string zero_key(const std::shared_ptr<const std::vector<uint8_t>>& z) {
  if(!z) return "-";
  uint64_t h = 1469598103934665603ull, n = 0;
  for(uint8_t x: *z) {
    h = (h ^ x) * 1099511628211ull;
    n += x;
  }
  return std::to_string(n) + ":" + std::to_string(h);
}

void Sched::prepare_mult(Op& op) {
  if(op.wl) return;
  const std::string sig = signature(op) + "|owner " + std::to_string(rank) + "/" + std::to_string(nranks) +
                          "|z " + zero_key(op.za) + " " + zero_key(op.zb);
  auto              pit = plan_cache.find(sig);
  if(pit == plan_cache.end()) {
    auto plan        = std::make_shared<Plan>();
    plan->lc         = classify(op.lhs.labels.data(), (int) op.lhs.labels.size(), op.a.labels.data(),
                                (int) op.a.labels.size(), op.b.labels.data(), (int) op.b.labels.size());
    plan->mode       = ctx->mode;
    plan->err_target = ctx->err_target;
    plan->nslices    = ctx->nslices;
    plan_cache[sig]  = plan;
    wl_cache[sig]    = build_mult_worklist(op, plan->lc, true, rank, nranks);
    pit              = plan_cache.find(sig);
  }
  op.plan = pit->second;
  op.wl   = wl_cache[sig];
}

// Assignment C = alpha * A * B, queued as Set(0) + Mult (MultOp::canonicalize,
// multop.hpp:255-269), on one rank: the contraction kernel (FP64, or the split kernels'
// epilogue) stores its result into the output blocks of groups with tasks (every
// element of those blocks is written once), and the Set zeroes only the blocks of
// groups without tasks.  Saves the fill of C and the read (or the atomic add) of every
// C element.
void Sched::fuse_assign(Op& set, Op& mult) {
  prepare_mult(mult);
  mult.store = true;
  if(set.set_blocks) return; // decided when this op first ran
  set.fill_key = "F|" + signature(mult) + "|owner " + std::to_string(rank) + "/" + std::to_string(nranks);
  auto blocks = std::make_shared<std::vector<int64_t>>();
  for(const auto& g: mult.wl->groups) {
    if(g.task_begin != g.task_end) continue;
    int64_t n = 1;
    for(int i = 0; i < mult.lhs.t->nmodes; i++) n *= g.cdims[i];
    blocks->push_back(g.c_off);
    blocks->push_back(n);
  }
  set.fill_none  = blocks->empty();
  set.set_blocks = blocks;
}

// Autotuner: each candidate (the FP64 kernel, the split-INT8 kernel at output tile
// widths 80 / 64 / 48 where the slice count allows) runs once to warm up and once
// timed with CUDA events, from the same saved copy of C; C is restored and the
// fastest candidate is kept for this signature and precision request.
void Sched::tune(Op& op, const std::string& key) {
  TuneChoice   ch;
  cudaStream_t st = ctx->stream;
  const LabelClasses& lc = op.plan->lc;
  std::vector<std::pair<int, int>> cand{{TB_MODE_FP64, 0}};
  const bool int8_kernel = !(lc.nbatch > 0 || lc.nar > 0 || lc.nbr > 0 || lc.nk == 0);
  if(int8_kernel) {
    const int S = ctx->nslices > 0 ? std::min(std::max(ctx->nslices, 3), 8) : int8_slices_for(ctx->err_target);
    for(int nt: {80, 64, 48})
      if(S * nt <= 512) cand.push_back({TB_MODE_INT8, nt});
  }
  if(cand.size() == 1) {
    ch.mode = TB_MODE_INT8; // nothing to choose: the INT8 request runs its FP64 route
    tune_cache[key] = ch;
    return;
  }
  Tensor&       C     = *op.lhs.t;
  const int64_t bytes = (int64_t) sizeof(double) * std::max<int64_t>(C.nelems, 1);
  double*       save  = static_cast<double*>(ctx->arena->allocate(bytes));
  TB_CUDA(cudaMemcpyAsync(save, C.data, bytes, cudaMemcpyDeviceToDevice, st));
  cudaEvent_t e0, e1;
  TB_CUDA(cudaEventCreate(&e0));
  TB_CUDA(cudaEventCreate(&e1));
  double best = 1e300;
  for(const auto& c: cand) {
    op.plan->mode   = c.first;
    op.plan->tile_n = c.second;
    float ms        = 0;
    for(int rep = 0; rep < 2; rep++) {
      TB_CUDA(cudaMemcpyAsync(C.data, save, bytes, cudaMemcpyDeviceToDevice, st));
      TB_CUDA(cudaEventRecord(e0, st));
      run_contract(*op.plan, *op.wl, op.alpha, op.a.t->data, op.b.t->data, C.data, st, ctx->arena.get());
      TB_CUDA(cudaEventRecord(e1, st));
      TB_CUDA(cudaEventSynchronize(e1));
      TB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    }
    ch.modes.push_back(c.first);
    ch.tiles.push_back(c.second);
    ch.ms.push_back(ms);
    if(ms < best) {
      best      = ms;
      ch.mode   = c.first;
      ch.tile_n = c.second;
    }
  }
  TB_CUDA(cudaMemcpyAsync(C.data, save, bytes, cudaMemcpyDeviceToDevice, st));
  TB_CUDA(cudaStreamSynchronize(st));
  ctx->arena->deallocate(save);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  tune_cache[key] = ch;
}

double* Sched::scalars() {
  if(!d_scalars) {
    TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&d_scalars), sizeof(double) * (kSlots + 1024)));
    TB_CUDA(cudaMemset(d_scalars, 0, sizeof(double) * (kSlots + 1024)));
  }
  return d_scalars;
}

Sched::~Sched() {
  if(d_scalars || !temps.empty()) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
  }
  if(d_scalars) cudaFree(d_scalars);
  for(auto& kv: temps)
    if(kv.second && kv.second->data) ctx->arena->deallocate(kv.second->data);
}

// Block table of a denominator op over t's admitted blocks: packed offset, dims and
// the root orbital index of each mode's first element (uploaded once).
void DenomSpec::build(const Tensor& T, const std::shared_ptr<Ctx>& c, const std::vector<int64_t>* only) {
  std::vector<DenomBlock> blocks;
  std::vector<int64_t>    id(T.nmodes);
  for(size_t bi = 0; bi < T.keys.size(); bi++) {
    if(only && !std::binary_search(only->begin(), only->end(), T.offsets[bi])) continue;
    int64_t key = T.keys[bi]; // block id in each mode's own tile numbering
    for(int m = T.nmodes - 1; m >= 0; m--) {
      const int64_t n = T.tis[m]->ntiles();
      id[m]           = key % n;
      key /= n;
    }
    DenomBlock b{};
    b.off = T.offsets[bi];
    for(int m = 0; m < T.nmodes; m++) {
      const int64_t r = T.tis[m]->tiles[id[m]]; // root tile
      b.dims[m]       = T.tis[m]->root->offsets[r + 1] - T.tis[m]->root->offsets[r];
      b.first[m]      = T.tis[m]->root->offsets[r];
      TB_EXPECTS(b.first[m] + b.dims[m] <= (int64_t) eps.size(), "orbital energies shorter than the index space");
    }
    blocks.push_back(b);
  }
  std::vector<DenomUnit> units;
  for(size_t bi = 0; bi < blocks.size(); bi++) {
    int64_t nrow = 1;
    for(int m = 0; m + 1 < T.nmodes; m++) nrow *= blocks[bi].dims[m];
    const int64_t ncol = blocks[bi].dims[T.nmodes - 1];
    const int64_t step = std::min<int64_t>(kDenomUnitRows, std::max<int64_t>(1, kDenomUnitElems / ncol));
    TB_EXPECTS(step * ncol < (1ll << 31), "denominator unit too large");
    for(int64_t r0 = 0; r0 < nrow; r0 += step)
      units.push_back(DenomUnit{(int32_t) bi, (int32_t) std::min(step, nrow - r0), r0});
  }
  TB_EXPECTS(units.size() < (1ull << 31), "too many denominator work units");
  ctx     = c;
  nblocks = (int) blocks.size();
  nunits  = (int) units.size();
  TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&d_eps), sizeof(double) * std::max<size_t>(eps.size(), 1)));
  TB_CUDA(cudaMemcpy(d_eps, eps.data(), sizeof(double) * eps.size(), cudaMemcpyHostToDevice));
  TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&d_blocks), sizeof(DenomBlock) * std::max<size_t>(blocks.size(), 1)));
  if(!blocks.empty())
    TB_CUDA(cudaMemcpy(d_blocks, blocks.data(), sizeof(DenomBlock) * blocks.size(), cudaMemcpyHostToDevice));
  TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&d_units), sizeof(DenomUnit) * std::max<size_t>(units.size(), 1)));
  if(!units.empty())
    TB_CUDA(cudaMemcpy(d_units, units.data(), sizeof(DenomUnit) * units.size(), cudaMemcpyHostToDevice));
  TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&d_part), sizeof(double) * std::max<size_t>(units.size(), 1)));
}

EnergySpec::~EnergySpec() {
  if(ctx) cudaSetDevice(ctx->device);
  if(args.estart) cudaFree(const_cast<int32_t*>(args.estart));
  if(args.part) cudaFree(args.part);
}

// The energy epilogue's device state for a Mult over its work list (see EnergySpec).
static std::shared_ptr<EnergySpec> build_energy(const Op& op, const LabelClasses& lc, const std::shared_ptr<Ctx>& ctx) {
  const Tensor&   C  = *op.lhs.t;
  const WorkList& wl = *op.wl;
  const int       nc = C.nmodes;
  auto            es = std::make_shared<EnergySpec>();
  es->ctx            = ctx;
  std::vector<int32_t> est(std::max<size_t>(wl.groups.size() * nc, 1), 0);
  std::vector<int64_t> rest;
  for(size_t gi = 0; gi < wl.groups.size(); gi++) {
    const DevGroup& g = wl.groups[gi];
    auto            o = std::lower_bound(C.offsets.begin(), C.offsets.end(), g.c_off);
    TB_EXPECTS(o != C.offsets.end() && *o == g.c_off, "energy epilogue: output group is not a stored block");
    if(g.task_begin == g.task_end) {
      rest.push_back(g.c_off);
      continue;
    }
    int64_t key = C.keys[o - C.offsets.begin()];
    int64_t id[kMaxModes];
    for(int m = nc - 1; m >= 0; m--) {
      id[m] = key % C.tis[m]->ntiles();
      key /= C.tis[m]->ntiles();
    }
    for(int m = 0; m < nc; m++) {
      const int64_t first = C.tis[m]->root->offsets[C.tis[m]->tiles[id[m]]];
      TB_EXPECTS(first + g.cdims[m] <= (int64_t) op.denom->eps.size(),
                 "orbital energies shorter than the index space");
      est[gi * nc + m] = (int32_t) first;
    }
    // partial sums: 8 warps per output tile, tiles at least 128 x 48 (every kernel's)
    int64_t M = 1, N = 1, Bt = 1;
    for(int j = 0; j < lc.nm; j++) M *= g.cdims[lc.m_c[j]];
    for(int j = 0; j < lc.nn; j++) N *= g.cdims[lc.n_c[j]];
    for(int j = 0; j < lc.nbatch; j++) Bt *= g.cdims[lc.batch_c[j]];
    es->npart += 8 * Bt * ((M + 127) / 128) * ((N + 47) / 48);
  }
  int32_t* d_est = nullptr;
  TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&d_est), sizeof(int32_t) * est.size()));
  es->args.estart = d_est;
  TB_CUDA(cudaMemcpy(d_est, est.data(), sizeof(int32_t) * est.size(), cudaMemcpyHostToDevice));
  TB_CUDA(cudaMalloc(reinterpret_cast<void**>(&es->args.part), sizeof(double) * std::max<int64_t>(es->npart, 1)));
  std::sort(rest.begin(), rest.end());
  if(!op.denom->d_eps) op.denom->build(C, ctx, &rest); // eps on the device (and the blocks for `rest`)
  es->args.eps = op.denom->d_eps;
  for(int m = 0; m < nc; m++) es->args.sg[m] = op.denom->signs[m];
  if(!rest.empty()) es->rest = op.denom;
  return es;
}

DenomSpec::~DenomSpec() {
  if(ctx) cudaSetDevice(ctx->device);
  if(d_eps) cudaFree(d_eps);
  if(d_blocks) cudaFree(d_blocks);
  if(d_part) cudaFree(d_part);
  if(d_units) cudaFree(d_units);
}

Graph::~Graph() {
  if(!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if(exec) cudaGraphExecDestroy(exec);
  if(graph) cudaGraphDestroy(graph);
  pool.release();
}

// A contraction with a lambda operand, batch by batch along the lambda tensor's first
// mode (see tb_tensor_create_lambda): consecutive tiles of that mode's label space
// whose admitted blocks fit the batch budget are materialised into scratch (one batch
// tensor per range, cached with the scheduler so that plans and work lists are too),
// the contraction runs over them with the first-mode label restricted to those tiles
// in every operand, and the scratch is released in stream order.
void Sched::run_lambda_mult(Op& op) {
  TB_EXPECTS(!(op.a.t->is_lambda() && op.b.t->is_lambda()), "a contraction of two lambda tensors is not supported");
  const bool on_a = op.a.t->is_lambda();
  Labeled&   X    = on_a ? op.a : op.b;
  Tensor&    L    = *X.t;
  TB_EXPECTS(L.nmodes >= 1, "a lambda tensor needs at least one mode");
  op.lhs.t->require_allocated();
  (on_a ? op.b : op.a).t->require_allocated();
  const int                   lab0 = X.labels[0];
  const std::shared_ptr<TIS>& sp0  = X.ltis[0];
  // elements of L's stored blocks per tile of the first mode's label space
  std::vector<int64_t> of_tile(L.tis[0]->ntiles(), -1); // L tile -> index in sp0
  for(int64_t k = 0; k < sp0->ntiles(); k++) {
    const int64_t t = L.tis[0]->find_root(sp0->tiles[k]);
    TB_EXPECTS(t >= 0, "label tile is not a tile of the lambda tensor's index space");
    of_tile[t] = k;
  }
  std::vector<int64_t> per(sp0->ntiles(), 0);
  for(size_t b = 0; b < L.keys.size(); b++) {
    const int64_t t0 = L.keys[b] / L.key_stride[0];
    const int64_t n  = (b + 1 < L.keys.size() ? L.offsets[b + 1] : L.nelems) - L.offsets[b];
    if(of_tile[t0] >= 0) per[of_tile[t0]] += n;
  }
  const int64_t budget = L.batch_bytes > 0 ? L.batch_bytes
                                           : std::max<int64_t>(64 << 20, (ctx->arena->capacity() - ctx->arena->used()) / 4);
  double              flops = 0, flops_run = 0, split_ms = 0, gemm_ms = 0, int8_ops = 0, int8_alg = 0;
  int                 smin = 99, smax = 0;
  const cudaStream_t  st = ctx->stream;
  for(int64_t k0 = 0; k0 < sp0->ntiles();) {
    int64_t k1 = k0 + 1, bytes = 8 * per[k0];
    while(k1 < sp0->ntiles() && bytes + 8 * per[k1] <= budget) bytes += 8 * per[k1++];
    const std::string key = std::to_string(L.serial.v) + "|" + std::to_string(sp0->serial.v) + "|" +
                            std::to_string(k0) + "-" + std::to_string(k1);
    auto& hb = lambda_batches[key];
    if(!hb) {
      hb         = std::make_unique<tb_tensor_s>();
      hb->p      = std::make_unique<Tensor>();
      Tensor& B  = *hb->p;
      B.nmodes   = L.nmodes;
      B.tis      = L.tis;
      B.tis[0]   = tis_subrange(*sp0, k0, k1);
      B.has_spin = L.has_spin;
      std::copy(L.mask, L.mask + kMaxModes, B.mask);
      B.build_table();
    }
    Tensor& B = *hb->p;
    void*   storage = pinned ? pinned->get(8 * std::max<int64_t>(B.nelems, 1))
                             : ctx->arena->allocate(8 * std::max<int64_t>(B.nelems, 1));
    B.data = static_cast<double*>(storage);
    B.ctx  = ctx;
    if(L.lambda_batch) {
      if(!builder) {
        builder      = std::make_unique<tb_sched_s>();
        builder->p   = std::make_unique<Sched>();
        builder->p->ctx = ctx;
      }
      builder->p->pinned = pinned;
      const int rc = L.lambda_batch(hb.get(), k0, k1, builder.get(), L.lambda_user);
      if(rc != 0) {
        builder->p->ops.clear();
        builder->p->start = 0;
        fail(TB_ERR_INVALID, "lambda tensor batch builder returned status " + std::to_string(rc));
      }
      builder->p->execute(false);
      builder->p->pinned = nullptr;
      for(size_t i = builder->p->last_first; i < builder->p->ops.size(); i++) {
        const auto& bo = builder->p->ops[i];
        if(bo.kind == Op::Mult && bo.wl) {
          if(pinned) batch_lists.push_back(bo.wl);
          else if(deferred_checks) pending.push_back(bo.wl);
        }
      }
    }
    else {
      std::vector<int64_t> bid(B.nmodes), lid(B.nmodes), dims(B.nmodes);
      for(size_t b = 0; b < B.keys.size(); b++) {
        int64_t key2 = B.keys[b];
        for(int m = B.nmodes - 1; m >= 0; m--) {
          bid[m] = key2 % B.tis[m]->ntiles();
          key2 /= B.tis[m]->ntiles();
        }
        lid       = bid;
        lid[0]    = L.tis[0]->find_root(B.tis[0]->tiles[bid[0]]);
        int64_t n = 1;
        for(int m = 0; m < B.nmodes; m++) n *= (dims[m] = B.tis[m]->size(bid[m]));
        const int rc = L.lambda_block(lid.data(), L.nmodes, dims.data(), B.data + B.offsets[b], n, st, L.lambda_user);
        if(rc != 0) fail(TB_ERR_INVALID, "lambda tensor block function returned status " + std::to_string(rc));
      }
    }
    // the contraction over this batch: the first-mode label takes the batch's tiles
    Op sub   = op;
    sub.plan = nullptr;
    sub.wl   = nullptr;
    sub.za    = on_a ? nullptr : op.za; // what is known of the stored operand stays
    sub.zb    = on_a ? op.zb : nullptr;
    sub.store = false;
    (on_a ? sub.a : sub.b).t = &B;
    if(L.lambda_batch) { // blocks the builder's assignment left without contributions
      auto z = builder->p->last_zeros.find(&B);
      if(z != builder->p->last_zeros.end()) (on_a ? sub.za : sub.zb) = z->second;
    }
    for(Labeled* x: {&sub.lhs, &sub.a, &sub.b})
      for(size_t m = 0; m < x->labels.size(); m++)
        if(x->labels[m] == lab0) x->ltis[m] = B.tis[0];
    run(sub);
    if(sub.wl) {
      if(pinned) batch_lists.push_back(sub.wl);
      else if(deferred_checks) pending.push_back(sub.wl);
    }
    if(sub.plan) {
      const tb_stats& s = sub.plan->last;
      flops += s.flops;
      flops_run += s.flops_run;
      split_ms += s.split_ms;
      gemm_ms += s.gemm_ms;
      int8_ops += s.int8_ops;
      int8_alg += s.int8_ops_alg;
      smin = std::min(smin, s.slices_min);
      smax = std::max(smax, s.slices_max);
    }
    if(pinned) pinned->put(storage);
    else ctx->arena->deallocate(storage); // reusable by later work on the stream
    B.data = nullptr;
    k0     = k1;
  }
  op.plan                 = std::make_shared<Plan>();
  op.plan->last           = tb_stats{};
  op.plan->last.flops     = flops;
  op.plan->last.flops_run = flops_run;
  op.plan->last.split_ms  = split_ms;
  op.plan->last.gemm_ms   = gemm_ms;
  op.plan->last.int8_ops  = int8_ops;
  op.plan->last.int8_ops_alg = int8_alg;
  op.plan->last.slices_min = smax > 0 ? smin : 0;
  op.plan->last.slices_max = smax;
  op.plan->last.mode      = ctx->mode;
  op.flops                = flops;
}

// Updates the blocks known to be zero after `op` ran (see Sched::execute).
void Sched::note_zeros(const Op& op, std::map<const Tensor*, std::shared_ptr<std::vector<uint8_t>>>& szero) {
  Tensor* t = op.lhs.t;
  if(t == nullptr || op.kind == Op::Dot || op.kind == Op::DenomEnergy || op.kind == Op::SetScalar || op.energy) return;
  if(op.kind == Op::Set) {
    bool whole = op.is_assign && op.value == 0.0;
    for(int m = 0; whole && m < t->nmodes; m++) whole = op.lhs.ltis[m]->tiles == t->tis[m]->tiles;
    if(whole) szero[t] = std::make_shared<std::vector<uint8_t>>(t->keys.size(), 1);
    else szero.erase(t);
    return;
  }
  auto it = szero.find(t);
  if(it == szero.end()) return;
  if(op.kind != Op::Mult || !op.wl) {
    szero.erase(it);
    return;
  }
  auto next = std::make_shared<std::vector<uint8_t>>(*it->second);
  for(const auto& g: op.wl->groups) {
    if(g.task_begin == g.task_end) continue;
    auto o = std::lower_bound(t->offsets.begin(), t->offsets.end(), g.c_off);
    if(o != t->offsets.end() && *o == g.c_off) (*next)[o - t->offsets.begin()] = 0;
  }
  it->second = next;
}

void Sched::execute(bool profile) {
  TB_CUDA(cudaSetDevice(ctx->device));
  // keep only the ops about to run (the history of earlier executes is not needed:
  // plans and work lists live in the caches)
  ops.erase(ops.begin(), ops.begin() + (long) start);
  start      = 0;
  last_first = 0;
  prof_ms.clear();
  prof_flops.clear();
  prof_stats.clear();
  profiling = profile;
  std::vector<cudaEvent_t> ev;
  if(profile) {
    ev.resize(2 * (ops.size() - start));
    for(auto& e: ev) TB_CUDA(cudaEventCreate(&e));
  }
  // Blocks known to be zero by construction, per tensor, from the ops of this execute
  // so far (nothing is assumed about a tensor's contents at the start): an assignment
  // of zero makes every block zero, a contraction into the tensor clears the blocks of
  // its output groups that have tasks, any other write forgets what was known.  This
  // follows the op list's structure only, never the data, so a graph capture of the
  // same list makes the same decisions for every replay.
  std::map<const Tensor*, std::shared_ptr<std::vector<uint8_t>>> szero;
  auto known = [&](const Tensor* t) -> std::shared_ptr<const std::vector<uint8_t>> {
    auto it = szero.find(t);
    return it == szero.end() ? nullptr : it->second;
  };
  for(size_t i = start; i < ops.size(); i++) {
    if(profile) TB_CUDA(cudaEventRecord(ev[2 * (i - start)], ctx->stream));
    if(ops[i].kind == Op::Mult) {
      ops[i].za = known(ops[i].a.t);
      ops[i].zb = known(ops[i].b.t);
    }
    if(i + 1 < ops.size() && ops[i + 1].kind == Op::Mult) {
      ops[i + 1].za = known(ops[i + 1].a.t);
      ops[i + 1].zb = known(ops[i + 1].b.t);
    }
    if(nranks == 1 && i + 1 < ops.size() && ops[i].kind == Op::Set &&
       ops[i].is_assign && ops[i].value == 0.0 &&
       ops[i + 1].kind == Op::Mult && !ops[i + 1].energy && same_target(ops[i].lhs, ops[i + 1].lhs) &&
       ops[i + 1].a.t != ops[i].lhs.t && ops[i + 1].b.t != ops[i].lhs.t && // C read as an operand needs the fill
       !ops[i + 1].a.t->is_lambda() && !ops[i + 1].b.t->is_lambda())      // (a batched op adds batch by batch)
      fuse_assign(ops[i], ops[i + 1]);
    run(ops[i]);
    note_zeros(ops[i], szero);
    if(ops[i].kind == Op::Mult && deferred_checks && ops[i].wl) pending.push_back(ops[i].wl);
    if(!pinned) // (a captured graph orders its own ops)
      for(Tensor* t: {ops[i].lhs.t, ops[i].a.t, ops[i].b.t}) mark_used(t, ctx->stream);
    if(profile) {
      TB_CUDA(cudaEventRecord(ev[2 * (i - start) + 1], ctx->stream));
      prof_stats.push_back(ops[i].kind == Op::Mult && ops[i].plan ? ops[i].plan->last : tb_stats{});
    }
  }
  profiling  = false;
  last_zeros = std::move(szero);
  if(profile) {
    TB_CUDA(cudaStreamSynchronize(ctx->stream));
    for(size_t i = start; i < ops.size(); i++) {
      float ms = 0;
      TB_CUDA(cudaEventElapsedTime(&ms, ev[2 * (i - start)], ev[2 * (i - start) + 1]));
      prof_ms.push_back(ms);
      prof_flops.push_back(ops[i].flops);
    }
    for(auto& e: ev) cudaEventDestroy(e);
  }
  start = ops.size();
}

} // namespace tb
