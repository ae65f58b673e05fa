// tamm_b200/tamm.hpp — C++ front-end with TAMM's LabeledTensor / Scheduler API.
//
// Header-only; every class lowers to the runtime tier of the C ABI
// (include/tamm_b200.h).  Mirrors the user-facing names of TAMM
// (src/tamm/index_space.hpp, tiled_index_space.hpp, tensor.hpp, labeled_tensor.hpp,
// scheduler.hpp) so code written against TAMM's contraction API compiles with
// `#include "tamm_b200/tamm.hpp"`:
//
//   sch(r2(a, b, i, j) += v(a, b, c, d) * t2(c, d, i, j)).execute(ExecutionHW::GPU);
//
// Errors are reported as exceptions carrying the library's message (TAMM's
// EXPECTS / NOT_IMPLEMENTED convention); all tensors hold double.
#pragma once

#include "tamm_b200.h"

#include <array>
#include <cstdint>
#include <initializer_list>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace tamm {

class Error: public std::runtime_error {
public:
  int status;
  Error(int s, const std::string& m): std::runtime_error(m), status(s) {}
};

inline void check(int status) {
  if(status == TB_OK) return;
  char buf[1024];
  tb_last_error(buf, sizeof buf);
  throw Error(status, std::string(tb_status_string(status)) + ": " + buf);
}

enum class ExecutionHW { DEFAULT = 0, CPU = 1, GPU = 2 };

enum class Precision { FP64 = TB_MODE_FP64, INT8 = TB_MODE_INT8, BF16X3 = TB_MODE_BF16X3 };

struct Spin {
  int value;
  explicit Spin(int v): value(v) {}
};

struct Range {
  int64_t lo, hi;
};
inline Range range(int64_t lo, int64_t hi) { return Range{lo, hi}; }
inline Range range(int64_t n) { return Range{0, n}; }

using Tile = int64_t;

// ExecutionContext: one GPU, its stream and the stream-ordered device arena.
class ExecutionContext {
public:
  explicit ExecutionContext(int device = 0, int64_t pool_bytes = 0) {
    tb_ctx c = nullptr;
    check(tb_ctx_create(device, pool_bytes, &c));
    h_ = std::shared_ptr<tb_ctx_s>(c, [](tb_ctx x) { tb_ctx_destroy(x); });
  }
  void set_precision(Precision p, double err_target = 1e-11, int nslices = 0) {
    check(tb_ctx_set_precision(h_.get(), static_cast<int>(p), err_target, nslices));
  }
  void* stream() const {
    void* s = nullptr;
    check(tb_ctx_stream(h_.get(), &s));
    return s;
  }
  void flush_and_sync() const { check(tb_ctx_synchronize(h_.get())); }
  tb_ctx handle() const { return h_.get(); }

private:
  std::shared_ptr<tb_ctx_s> h_;
};

// IndexSpace{range(n), {{name, {ranges}}...}, {{Spin{s}, {ranges}}...}}
class IndexSpace {
public:
  using NamedRanges = std::vector<std::pair<std::string, std::vector<Range>>>;
  using SpinRanges  = std::vector<std::pair<Spin, std::vector<Range>>>;

  IndexSpace(Range r, const NamedRanges& named = {}, const SpinRanges& spin = {}) {
    if(r.lo != 0) throw Error(TB_ERR_INVALID, "IndexSpace ranges start at 0");
    std::vector<const char*> names;
    std::vector<int>         nn, sv, sn;
    std::vector<int64_t>     nr, sr;
    for(const auto& kv: named) {
      names.push_back(kv.first.c_str());
      nn.push_back((int) kv.second.size());
      for(const auto& x: kv.second) {
        nr.push_back(x.lo);
        nr.push_back(x.hi);
      }
    }
    for(const auto& kv: spin) {
      sv.push_back(kv.first.value);
      sn.push_back((int) kv.second.size());
      for(const auto& x: kv.second) {
        sr.push_back(x.lo);
        sr.push_back(x.hi);
      }
    }
    tb_is h = nullptr;
    check(tb_is_create(r.hi, (int) names.size(), names.data(), nn.data(), nr.data(), (int) sv.size(),
                       sv.data(), sn.data(), sr.data(), &h));
    h_ = std::shared_ptr<tb_is_s>(h, [](tb_is x) { tb_is_destroy(x); });
  }
  tb_is handle() const { return h_.get(); }

private:
  std::shared_ptr<tb_is_s> h_;
};

class TiledIndexSpace;

// TiledIndexLabel: a label bound to a tiled index space; labels compare by identity.
class TiledIndexLabel {
public:
  TiledIndexLabel() = default;
  TiledIndexLabel(std::shared_ptr<tb_tis_s> tis, int id): tis_(std::move(tis)), id_(id) {}
  tb_tis tis() const { return tis_.get(); }
  int    id() const { return id_; }
  const std::shared_ptr<tb_tis_s>& shared_tis() const { return tis_; }

private:
  std::shared_ptr<tb_tis_s> tis_;
  int                       id_ = 0;
};

inline int next_label_id() {
  static int n = 0;
  return ++n;
}

// TiledIndexSpace{is, tile} or TiledIndexSpace{is, tile_list}; tis("name") is the
// named subspace; TiledIndexSpace{tis, range(first, last)} a range of tiles.
class TiledIndexSpace {
public:
  TiledIndexSpace() = default;
  TiledIndexSpace(const IndexSpace& is, Tile tile) {
    tb_tis h = nullptr;
    check(tb_tis_create(is.handle(), tile, nullptr, 0, &h));
    wrap(h);
  }
  TiledIndexSpace(const IndexSpace& is, const std::vector<Tile>& tiles) {
    tb_tis h = nullptr;
    check(tb_tis_create(is.handle(), 0, tiles.data(), (int64_t) tiles.size(), &h));
    wrap(h);
  }
  TiledIndexSpace(const TiledIndexSpace& parent, Range tiles) {
    tb_tis h = nullptr;
    check(tb_tis_subrange(parent.handle(), tiles.lo, tiles.hi, &h));
    wrap(h);
  }
  TiledIndexSpace operator()(const std::string& name = "all") const {
    tb_tis h = nullptr;
    check(tb_tis_named(handle(), name.c_str(), &h));
    TiledIndexSpace t;
    t.wrap(h);
    return t;
  }
  int64_t num_tiles() const {
    int64_t n = 0;
    check(tb_tis_num_tiles(handle(), &n));
    return n;
  }
  std::vector<int64_t> tile_sizes() const {
    std::vector<int64_t> s(num_tiles());
    check(tb_tis_tiles(handle(), s.data(), nullptr, nullptr));
    return s;
  }
  int64_t tile_size(int64_t i) const { return tile_sizes().at(i); }
  std::vector<int> spins() const {
    std::vector<int> s(num_tiles());
    check(tb_tis_tiles(handle(), nullptr, s.data(), nullptr));
    return s;
  }
  TiledIndexLabel label(const std::string& = "") const { return TiledIndexLabel(h_, next_label_id()); }
  template<size_t N>
  auto labels(const std::string& name = "all") const {
    const TiledIndexSpace sp = name == "all" ? *this : (*this)(name);
    std::array<TiledIndexLabel, N> out;
    for(auto& l: out) l = sp.label();
    return array_to_tuple(out, std::make_index_sequence<N>{});
  }
  tb_tis handle() const { return h_.get(); }
  const std::shared_ptr<tb_tis_s>& shared() const { return h_; }
  static TiledIndexSpace from_shared(std::shared_ptr<tb_tis_s> h) {
    TiledIndexSpace t;
    t.h_ = std::move(h);
    return t;
  }

private:
  void wrap(tb_tis h) { h_ = std::shared_ptr<tb_tis_s>(h, [](tb_tis x) { tb_tis_destroy(x); }); }
  template<size_t N, size_t... I>
  static auto array_to_tuple(const std::array<TiledIndexLabel, N>& a, std::index_sequence<I...>) {
    return std::make_tuple(a[I]...);
  }
  std::shared_ptr<tb_tis_s> h_;
};

template<typename T>
class Tensor;

// One operand of an op: tensor + per-mode label keys (a TiledIndexLabel, a string
// label, or the tensor's own mode for T()).
struct LabelKey {
  int         kind = 0; // 0 tiled label, 1 string, 2 own mode
  int         id   = 0;
  std::string name;
  tb_tis      tis = nullptr;
};

class LabeledTensorBase {
public:
  tb_tensor             tensor = nullptr;
  std::vector<LabelKey> keys;
};

template<typename T>
class LabeledTensor;

struct Product {
  double                         alpha = 1.0;
  std::vector<LabeledTensorBase> factors;
};

inline Product operator*(double s, const Product& p) {
  Product r = p;
  r.alpha *= s;
  return r;
}
inline Product operator*(const Product& p, double s) { return s * p; }

struct OpSpec {
  LabeledTensorBase lhs;
  bool              is_assign = false;
  double            sign      = 1.0;
  bool              scalar    = false;
  double            value     = 0.0;
  Product           rhs;
};

template<typename T>
class LabeledTensor: public LabeledTensorBase {
public:
  OpSpec operator=(double v) const { return scalar_op(v, true, 1.0); }
  OpSpec operator+=(double v) const { return scalar_op(v, false, 1.0); }
  OpSpec operator-=(double v) const { return scalar_op(v, false, -1.0); }
  OpSpec operator=(const Product& p) const { return prod_op(p, true, 1.0); }
  OpSpec operator+=(const Product& p) const { return prod_op(p, false, 1.0); }
  OpSpec operator-=(const Product& p) const { return prod_op(p, false, -1.0); }
  OpSpec operator=(const LabeledTensor& o) const { return prod_op(Product{1.0, {o}}, true, 1.0); }
  OpSpec operator+=(const LabeledTensor& o) const { return prod_op(Product{1.0, {o}}, false, 1.0); }
  OpSpec operator-=(const LabeledTensor& o) const { return prod_op(Product{1.0, {o}}, false, -1.0); }

private:
  OpSpec scalar_op(double v, bool assign, double sign) const {
    OpSpec s;
    s.lhs       = *this;
    s.is_assign = assign;
    s.sign      = sign;
    s.scalar    = true;
    s.value     = v;
    return s;
  }
  OpSpec prod_op(const Product& p, bool assign, double sign) const {
    OpSpec s;
    s.lhs       = *this;
    s.is_assign = assign;
    s.sign      = sign;
    s.rhs       = p;
    return s;
  }
};

template<typename T>
Product operator*(const LabeledTensor<T>& a, const LabeledTensor<T>& b) {
  return Product{1.0, {a, b}};
}
template<typename T>
Product operator*(double s, const LabeledTensor<T>& a) {
  return Product{s, {a}};
}
template<typename T>
Product operator*(const Product& p, const LabeledTensor<T>& b) {
  Product r = p;
  r.factors.push_back(b);
  return r;
}

// Tensor<double>{tis...}, Tensor<double>{{tis...}, {nupper, nlower}}
template<typename T>
class Tensor {
  static_assert(std::is_same_v<T, double>, "tamm_b200 tensors hold double");

public:
  Tensor() { create({}, nullptr); } // Tensor<T>{}: a scalar (0-mode) tensor
  Tensor(std::initializer_list<TiledIndexSpace> tis) { create(std::vector<TiledIndexSpace>(tis), nullptr); }
  Tensor(std::initializer_list<TiledIndexLabel> labels) {
    std::vector<TiledIndexSpace> v;
    for(const auto& l: labels) v.push_back(TiledIndexSpace::from_shared(l.shared_tis()));
    create(v, nullptr);
  }
  Tensor(const std::vector<TiledIndexSpace>& tis, std::pair<int, int> spin_sizes) {
    std::vector<int> mask;
    for(size_t i = 0; i < tis.size(); i++)
      mask.push_back((int) i < spin_sizes.first ? 0 : ((int) i < spin_sizes.first + spin_sizes.second ? 1 : 2));
    create(tis, &mask);
  }
  Tensor(const std::vector<TiledIndexSpace>& tis, std::initializer_list<int> spin_sizes):
    Tensor(tis, std::make_pair(*spin_sizes.begin(), spin_sizes.size() > 1 ? *(spin_sizes.begin() + 1)
                                                                           : (int) tis.size() - *spin_sizes.begin())) {}

  template<typename... L>
  LabeledTensor<T> operator()(const L&... labels) const {
    LabeledTensor<T> lt;
    lt.tensor = h_.get();
    (lt.keys.push_back(key(labels)), ...);
    if constexpr(sizeof...(L) == 0) {
      for(int i = 0; i < nmodes_; i++) {
        LabelKey k;
        k.kind = 2;
        k.id   = i;
        lt.keys.push_back(k);
      }
    }
    if(lt.keys.size() == 1 && lt.keys[0].kind == 1 && nmodes_ != 1) {
      // "a,b,i,j" string labels
      std::vector<LabelKey> ks;
      std::stringstream     ss(lt.keys[0].name);
      std::string           tok;
      while(std::getline(ss, tok, ',')) {
        LabelKey k;
        k.kind = 1;
        k.name = tok;
        ks.push_back(k);
      }
      lt.keys = ks;
    }
    if((int) lt.keys.size() != nmodes_) throw Error(TB_ERR_INVALID, "wrong number of labels for this tensor");
    return lt;
  }

  void allocate(const ExecutionContext& ec) { check(tb_tensor_allocate(h_.get(), ec.handle())); }
  void deallocate() { check(tb_tensor_deallocate(h_.get())); }
  int  num_modes() const { return nmodes_; }
  int64_t size() const {
    int     nm = 0;
    int64_t nb = 0, ne = 0;
    check(tb_tensor_info(h_.get(), &nm, &nb, &ne));
    return ne;
  }
  bool is_non_zero(const std::vector<int64_t>& blockid) const {
    int r = 0;
    check(tb_tensor_is_non_zero(h_.get(), blockid.data(), &r));
    return r != 0;
  }
  std::vector<double> get(const std::vector<int64_t>& blockid) const {
    int64_t n = 0;
    check(tb_tensor_block_size(h_.get(), blockid.data(), &n));
    std::vector<double> buf(n);
    check(tb_tensor_get(h_.get(), blockid.data(), buf.data(), n));
    return buf;
  }
  void put(const std::vector<int64_t>& blockid, const std::vector<double>& buf) {
    check(tb_tensor_put(h_.get(), blockid.data(), buf.data(), (int64_t) buf.size()));
  }
  void add(const std::vector<int64_t>& blockid, const std::vector<double>& buf) {
    check(tb_tensor_add(h_.get(), blockid.data(), buf.data(), (int64_t) buf.size()));
  }
  std::vector<double> read() const {
    std::vector<double> v(size());
    check(tb_tensor_read(h_.get(), v.data(), (int64_t) v.size()));
    return v;
  }
  void write(const std::vector<double>& v) { check(tb_tensor_write(h_.get(), v.data(), (int64_t) v.size())); }
  // contents constant until cleared; contractions skip tasks over its all-zero blocks
  void set_read_only(bool on = true) { check(tb_tensor_set_read_only(h_.get(), on ? 1 : 0)); }
  tb_tensor handle() const { return h_.get(); }

private:
  LabelKey key(const TiledIndexLabel& l) const {
    LabelKey k;
    k.kind = 0;
    k.id   = l.id();
    k.tis  = l.tis();
    return k;
  }
  LabelKey key(const std::string& s) const {
    LabelKey k;
    k.kind = 1;
    k.name = s;
    return k;
  }
  LabelKey key(const char* s) const { return key(std::string(s)); }
  void create(const std::vector<TiledIndexSpace>& tis, const std::vector<int>* mask) {
    std::vector<tb_tis> hs;
    for(const auto& t: tis) {
      hs.push_back(t.handle());
      keep_.push_back(t.shared());
    }
    tb_tensor h = nullptr;
    check(tb_tensor_create((int) hs.size(), hs.data(), mask ? mask->data() : nullptr, &h));
    h_      = std::shared_ptr<tb_tensor_s>(h, [](tb_tensor x) { tb_tensor_destroy(x); });
    nmodes_ = (int) hs.size();
  }
  std::shared_ptr<tb_tensor_s>           h_;
  std::vector<std::shared_ptr<tb_tis_s>> keep_;
  int                                    nmodes_ = 0;
  friend class Scheduler;
};

// tamm::norm (src/tamm/tamm_utils.hpp:1180-1200): sqrt of the sum of squares of
// every stored element, reduced on the device.
template<typename T>
double norm(const Tensor<T>& t) {
  double r = 0.0;
  check(tb_tensor_norm(t.handle(), &r));
  return r;
}

// Scheduler{ec}: sch(op)(op)...execute(hw, profile)
class Scheduler {
public:
  explicit Scheduler(const ExecutionContext& ec): ec_(ec) {
    tb_sched s = nullptr;
    check(tb_sched_create(ec.handle(), &s));
    h_ = std::shared_ptr<tb_sched_s>(s, [](tb_sched x) { tb_sched_destroy(x); });
  }

  template<typename... Ts>
  Scheduler& allocate(Ts&... tensors) {
    (tensors.allocate(ec_), ...);
    return *this;
  }
  template<typename... Ts>
  Scheduler& deallocate(Ts&... tensors) {
    (tensors.deallocate(), ...);
    return *this;
  }

  Scheduler& operator()(const OpSpec& op, const std::string& = "", ExecutionHW = ExecutionHW::DEFAULT) {
    std::map<std::string, int> ids;
    std::vector<Lowered>       keep;
    tb_labeled                 lhs = lower(op.lhs, ids, keep);
    if(op.scalar) {
      check(tb_sched_set(h_.get(), lhs, op.sign * op.value, op.is_assign ? 1 : 0));
      return *this;
    }
    const double alpha = op.sign * op.rhs.alpha;
    if(op.rhs.factors.size() == 1) {
      tb_labeled a = lower(op.rhs.factors[0], ids, keep);
      check(tb_sched_add(h_.get(), lhs, alpha, a, op.is_assign ? 1 : 0));
    }
    else if(op.rhs.factors.size() == 2) {
      tb_labeled a = lower(op.rhs.factors[0], ids, keep);
      tb_labeled b = lower(op.rhs.factors[1], ids, keep);
      check(tb_sched_mult(h_.get(), lhs, alpha, a, b, op.is_assign ? 1 : 0));
    }
    else throw Error(TB_ERR_INVALID, "an op has one or two tensor factors");
    return *this;
  }

  // MapOp family: lhs = fn(rhs) element by element (TB_MAP_*; rhs has lhs's labels,
  // may be lhs itself); exact_copy (Scheduler::exact_copy, scheduler.hpp:461).
  Scheduler& map(const LabeledTensorBase& lhs, const LabeledTensorBase& rhs, int fn, double p = 0.0) {
    std::map<std::string, int> ids;
    std::vector<Lowered>       keep;
    tb_labeled                 l = lower(lhs, ids, keep);
    tb_labeled                 r = lower(rhs, ids, keep);
    check(tb_sched_map(h_.get(), l, r, fn, p));
    return *this;
  }
  Scheduler& exact_copy(const LabeledTensorBase& lhs, const LabeledTensorBase& rhs) {
    return map(lhs, rhs, TB_MAP_COPY);
  }

  void execute(ExecutionHW hw = ExecutionHW::DEFAULT, bool profile = false) {
    check(tb_sched_execute(h_.get(), static_cast<int>(hw), profile ? 1 : 0));
  }

  ExecutionContext& ec() { return ec_; }

private:
  friend class Tape;
  struct Lowered {
    std::shared_ptr<std::vector<int>>    labels;
    std::shared_ptr<std::vector<tb_tis>> spaces;
  };
  // per-op int labels: equal keys get equal ints (MultOp::fillin_int_labels)
  static tb_labeled lower(const LabeledTensorBase& lt, std::map<std::string, int>& ids,
                          std::vector<Lowered>& keep) {
    Lowered l{std::make_shared<std::vector<int>>(), std::make_shared<std::vector<tb_tis>>()};
    for(const auto& k: lt.keys) {
      std::string key = k.kind == 0 ? "L" + std::to_string(k.id)
                                    : (k.kind == 1 ? "S" + k.name : "M" + std::to_string(k.id));
      auto it = ids.find(key);
      if(it == ids.end()) it = ids.emplace(key, -(int) (ids.size() + 1)).first;
      l.labels->push_back(it->second);
      l.spaces->push_back(k.kind == 0 ? k.tis : nullptr);
    }
    keep.push_back(l);
    return tb_labeled{lt.tensor, l.labels->data(), l.spaces->data()};
  }
  ExecutionContext            ec_;
  std::shared_ptr<tb_sched_s> h_;
};

// Forward/backward Functions on a Scheduler (no counterpart in TAMM; tb_tape_* in
// tamm_b200.h).  Contract's backward is the pair of swapped-operand contractions
// dA += alpha * dC * B, dB += alpha * A * dC; Dot's a pair of permuted adds; the
// objective is the sum of the Dot values.  Contract outputs beyond the memory budget
// are freed at the start of backward() and recomputed when needed.
//
//   Tape tape{ec};
//   tape.leaf(t2, g);                                       // g += dE/dt2
//   tape.contract(X(a, b, i, j), v(a, b, c, d) * t2(c, d, i, j));
//   double E = tape.dot(w(i, j, a, b), t2(a, b, i, j)) + tape.dot(t2(a, b, i, j), X(a, b, i, j), 0.25);
//   tape.backward();
class Tape {
public:
  explicit Tape(const ExecutionContext& ec, int64_t budget_bytes = INT64_MAX): ec_(ec) {
    tb_tape t = nullptr;
    check(tb_tape_create(ec.handle(), budget_bytes, &t));
    h_ = std::shared_ptr<tb_tape_s>(t, [](tb_tape x) { tb_tape_destroy(x); });
  }

  template<typename T>
  Tape& leaf(const Tensor<T>& x, const Tensor<T>& grad) {
    check(tb_tape_leaf(h_.get(), x.handle(), grad.handle()));
    return *this;
  }

  template<typename T>
  Tape& contract(const LabeledTensor<T>& y, const Product& p) {
    if(p.factors.size() != 2) throw Error(TB_ERR_INVALID, "contract takes a product of two labelled tensors");
    std::map<std::string, int>    ids;
    std::vector<Scheduler::Lowered> keep;
    tb_labeled                    ly = Scheduler::lower(y, ids, keep);
    tb_labeled                    la = Scheduler::lower(p.factors[0], ids, keep);
    tb_labeled                    lb = Scheduler::lower(p.factors[1], ids, keep);
    check(tb_tape_contract(h_.get(), ly, p.alpha, la, lb));
    return *this;
  }

  double dot(const LabeledTensorBase& p, const LabeledTensorBase& q, double alpha = 1.0) {
    std::map<std::string, int>    ids;
    std::vector<Scheduler::Lowered> keep;
    tb_labeled                    lp = Scheduler::lower(p, ids, keep);
    tb_labeled                    lq = Scheduler::lower(q, ids, keep);
    double                        v  = 0.0;
    check(tb_tape_dot(h_.get(), alpha, lp, lq, &v));
    return v;
  }

  void backward() { check(tb_tape_backward(h_.get())); }
  void reset() { check(tb_tape_reset(h_.get())); }
  int64_t recomputed() const {
    int64_t r = 0;
    check(tb_tape_info(h_.get(), nullptr, nullptr, nullptr, &r));
    return r;
  }

private:
  ExecutionContext           ec_;
  std::shared_ptr<tb_tape_s> h_;
};

} // namespace tamm
