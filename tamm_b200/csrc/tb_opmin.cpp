// Operation minimisation of multi-factor products and their execution as a sequence of
// binary contractions (TAMM's OpMin / OpExecutor, src/tamm/opmin.hpp:395-660,
// src/tamm/op_executor.hpp).
//
// lhs (=|+=) alpha * F_0 * F_1 * ... * F_(n-1): the binary contraction tree is chosen by
// dynamic programming over the subsets of the factors, with the cost model of
// opmin::Optimizer (opmin.hpp:455-530): a subset x needs the labels of x that occur
// outside x or on the left-hand side (required), combining disjoint x and y costs the
// product of the dense extents of required(x) | required(y), and the tree of least
// total cost wins, ties to the pair met first when subsets are visited by size, then
// by value (enumerate_power_set_minus_empty_set, opmin.hpp:60-81).  Every inner node
// becomes an intermediate tensor over its required labels (label order ascending, no
// spin symmetry, so every block is stored), assigned as Set(0) + Mult; the root
// updates the left-hand side.  Intermediates belong to the Scheduler and are reused
// when the same product is queued again.
#include "tb_runtime.hpp"

#include <algorithm>
#include <functional>
#include <limits>
#include <map>

namespace tb {

namespace {

struct OpminTree {
  int                   n = 0;
  std::vector<int64_t>  child1, child2; // per subset; -1 for a leaf
  std::vector<uint64_t> required;       // label bits a subset still needs
  std::vector<double>   cost;
  std::vector<int>      label_of_bit;
};

OpminTree optimize(const std::vector<std::vector<int>>& factors, const std::vector<int>& lhs,
                   const std::map<int, double>& extent) {
  OpminTree T;
  const int n = (int) factors.size();
  TB_EXPECTS(n >= 1 && n <= 20, "opmin takes 1..20 factors");
  T.n = n;
  std::vector<int> labels; // ascending: bit b names labels[b]
  for(const auto& f: factors) labels.insert(labels.end(), f.begin(), f.end());
  labels.insert(labels.end(), lhs.begin(), lhs.end());
  std::sort(labels.begin(), labels.end());
  labels.erase(std::unique(labels.begin(), labels.end()), labels.end());
  TB_EXPECTS(labels.size() <= 64, "opmin takes at most 64 distinct labels");
  T.label_of_bit = labels;
  auto bit = [&](int l) { return uint64_t(1) << (std::lower_bound(labels.begin(), labels.end(), l) - labels.begin()); };
  const uint64_t full = (uint64_t(1) << n) - 1;
  std::vector<uint64_t> avail(full + 1, 0);
  T.child1.assign(full + 1, -1);
  T.child2.assign(full + 1, -1);
  T.required.assign(full + 1, 0);
  T.cost.assign(full + 1, std::numeric_limits<double>::max());
  uint64_t lhs_bits = 0;
  for(int l: lhs) lhs_bits |= bit(l);
  for(int i = 0; i < n; i++) {
    T.cost[uint64_t(1) << i] = 0;
    for(int l: factors[i]) avail[uint64_t(1) << i] |= bit(l);
  }
  // subsets by size, then by value
  std::vector<uint64_t> order;
  for(int k = 1; k <= n; k++)
    for(uint64_t x = 1; x <= full; x++)
      if(__builtin_popcountll(x) == k) order.push_back(x);
  for(size_t a = 0; a < order.size(); a++) // availability of unions
    for(size_t b = 0; b < a; b++) avail[order[a] | order[b]] = avail[order[a]] | avail[order[b]];
  for(uint64_t x: order) T.required[x] = avail[x] & (avail[full & ~x] | lhs_bits);
  auto size_of = [&](uint64_t ids) {
    double s = 1;
    for(size_t b = 0; b < labels.size(); b++)
      if(ids >> b & 1) s *= extent.at(labels[b]);
    return s;
  };
  for(size_t a = 0; a < order.size(); a++) {
    const uint64_t x = order[a];
    for(size_t b = 0; b < a; b++) {
      const uint64_t y = order[b];
      if(x & y) continue;
      const double c = size_of(T.required[x] | T.required[y]) + T.cost[x] + T.cost[y];
      if(c < T.cost[x | y]) {
        T.cost[x | y]   = c;
        T.child1[x | y] = (int64_t) x;
        T.child2[x | y] = (int64_t) y;
      }
    }
  }
  return T;
}

// Labels of an operand (int labels) and the dense extent of each label's space.
void note_labels(const Labeled& x, std::map<int, double>& extent, std::map<int, std::shared_ptr<TIS>>& space) {
  for(size_t m = 0; m < x.labels.size(); m++) {
    const auto& s = x.ltis[m];
    double      e = 0;
    for(int64_t t = 0; t < s->ntiles(); t++) e += (double) s->size(t);
    extent[x.labels[m]] = e;
    if(!space.count(x.labels[m])) space[x.labels[m]] = s;
  }
}

OpminTree plan_of(const Labeled& lhs, const std::vector<Labeled>& f, std::map<int, std::shared_ptr<TIS>>& space) {
  std::map<int, double>         extent;
  std::vector<std::vector<int>> fl;
  note_labels(lhs, extent, space);
  for(const auto& x: f) {
    note_labels(x, extent, space);
    fl.push_back(x.labels);
  }
  return optimize(fl, lhs.labels, extent);
}

} // namespace

// Queues lhs (=|+=) alpha * prod(f) on the scheduler as binary contractions.
void queue_mult_n(Sched& s, const Labeled& lhs, double alpha, const std::vector<Labeled>& f, int is_assign,
                  const std::function<void(Op&&)>& push) {
  std::map<int, std::shared_ptr<TIS>> space;
  const OpminTree                     T    = plan_of(lhs, f, space);
  const uint64_t                      full = (uint64_t(1) << T.n) - 1;
  std::map<std::string, int>          seen; // intermediates of one signature in this product
  auto emit_mult = [&](const Labeled& c, double a, const Labeled& x, const Labeled& y, int assign) {
    if(assign) {
      Op set;
      set.kind      = Op::Set;
      set.lhs       = c;
      set.value     = 0.0;
      set.is_assign = 1;
      push(std::move(set));
    }
    Op op;
    op.kind  = Op::Mult;
    op.lhs   = c;
    op.a     = x;
    op.b     = y;
    op.alpha = a;
    (void) classify(op.lhs.labels.data(), (int) op.lhs.labels.size(), op.a.labels.data(), (int) op.a.labels.size(),
                    op.b.labels.data(), (int) op.b.labels.size());
    push(std::move(op));
  };
  std::function<Labeled(uint64_t)> node = [&](uint64_t x) -> Labeled {
    if(T.child1[x] < 0) return f[__builtin_ctzll(x)];
    const Labeled a = node((uint64_t) T.child1[x]), b = node((uint64_t) T.child2[x]);
    // intermediate over the required labels, ascending
    Labeled     t;
    std::string sig;
    std::vector<std::shared_ptr<TIS>> tis;
    for(size_t bt = 0; bt < T.label_of_bit.size(); bt++)
      if(T.required[x] >> bt & 1) {
        const int l = T.label_of_bit[bt];
        t.labels.push_back(l);
        tis.push_back(space.at(l));
        sig += std::to_string(space.at(l)->serial.v) + ",";
      }
    TB_EXPECTS(!tis.empty() && tis.size() <= kMaxModes, "opmin intermediate rank out of range");
    sig += "#" + std::to_string(seen[sig]++);
    auto& slot = s.temps[sig];
    if(!slot) {
      slot         = std::make_unique<Tensor>();
      slot->nmodes = (int) tis.size();
      slot->tis    = tis;
      slot->build_table();
      slot->data = static_cast<double*>(s.ctx->arena->allocate(sizeof(double) * std::max<int64_t>(slot->nelems, 1)));
      slot->ctx  = s.ctx;
    }
    t.t    = slot.get();
    t.ltis = tis;
    emit_mult(t, 1.0, a, b, 1);
    return t;
  };
  if(T.n == 1) {
    Op op;
    op.kind      = Op::Add;
    op.lhs       = lhs;
    op.a         = f[0];
    op.alpha     = alpha;
    op.is_assign = is_assign;
    push(std::move(op));
    return;
  }
  const Labeled a = node((uint64_t) T.child1[full]), b = node((uint64_t) T.child2[full]);
  emit_mult(lhs, alpha, a, b, is_assign);
}

// The chosen tree for tests and tools: the binary steps in execution order as (subset,
// subset) pairs of factor bit masks, and the total cost of the model.
void mult_n_order(const Labeled& lhs, const std::vector<Labeled>& f, std::vector<int64_t>& pairs, double& cost) {
  std::map<int, std::shared_ptr<TIS>> space;
  const OpminTree                     T    = plan_of(lhs, f, space);
  const uint64_t                      full = (uint64_t(1) << T.n) - 1;
  pairs.clear();
  std::function<void(uint64_t)> walk = [&](uint64_t x) {
    if(T.child1[x] < 0) return;
    walk((uint64_t) T.child1[x]);
    walk((uint64_t) T.child2[x]);
    pairs.push_back(T.child1[x]);
    pairs.push_back(T.child2[x]);
  };
  walk(full);
  cost = T.n > 1 ? T.cost[full] : 0.0;
}

} // namespace tb
