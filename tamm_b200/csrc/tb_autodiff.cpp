// Differentiation of contraction sequences: a tape of Functions on a Scheduler.
//
// TAMM has no automatic differentiation; this is the adjoint that coupled-cluster
// energy gradients need, built from the same MultOp / AddOp machinery:
//   Contract   y(Ly) = alpha * a(La) * b(Lb)        (forward: SetOp(0) + MultOp)
//     backward:  da(La) += alpha * dy(Ly) * b(Lb)   (the dy-weighted contractions over
//                db(Lb) += alpha * a(La) * dy(Ly)    the labels free in the other operand)
//   Dot        s = alpha * sum p(Lp) * q(Lq)        (q's modes matched to p's by label)
//     backward:  dp(Lp) += alpha * q(Lq),  dq(Lq) += alpha * p(Lp)
// The objective is the sum of the recorded Dot values.  Functions run eagerly on the
// tape's own Scheduler (its plan and work-list caches persist across evaluations),
// in the context's precision mode.
//
// Checkpointing: at the start of the backward sweep the Contract outputs are kept in
// recording order while their total size fits the memory budget; the others are
// freed and recomputed from their producer (itself recomputed if needed) when the
// sweep first needs their values.
#include "tb_api.hpp"
#include "tb_runtime.hpp"

#include <algorithm>
#include <set>

namespace tb {

namespace {

bool same_layout(const Tensor& x, const Tensor& y) {
  if(x.nmodes != y.nmodes || x.has_spin != y.has_spin || x.keys != y.keys || x.offsets != y.offsets) return false;
  for(int i = 0; i < x.nmodes; i++)
    if(x.tis[i]->root != y.tis[i]->root || x.tis[i]->tiles != y.tis[i]->tiles || x.mask[i] != y.mask[i])
      return false;
  return true;
}

bool full_spaces(const Labeled& l) {
  for(int i = 0; i < l.t->nmodes; i++)
    if(l.ltis[i]->root != l.t->tis[i]->root || l.ltis[i]->tiles != l.t->tis[i]->tiles) return false;
  return true;
}

double* arena_alloc(const std::shared_ptr<Ctx>& ctx, int64_t nelems) {
  return static_cast<double*>(ctx->arena->allocate(sizeof(double) * std::max<int64_t>(nelems, 1)));
}

std::unique_ptr<Tensor> clone_structure(const Tensor& x, const std::shared_ptr<Ctx>& ctx) {
  auto t      = std::make_unique<Tensor>();
  t->nmodes   = x.nmodes;
  t->tis      = x.tis;
  t->has_spin = x.has_spin;
  for(int i = 0; i < kMaxModes; i++) t->mask[i] = x.mask[i];
  t->build_table();
  t->data = arena_alloc(ctx, t->nelems);
  t->ctx  = ctx;
  return t;
}

Labeled relabel(const Labeled& l, Tensor* t) {
  Labeled r = l;
  r.t       = t;
  return r;
}

bool contains(const std::vector<int>& v, int x) { return std::find(v.begin(), v.end(), x) != v.end(); }

Op set_zero(const Labeled& l) {
  Op op;
  op.kind      = Op::Set;
  op.lhs       = l;
  op.value     = 0.0;
  op.is_assign = 1;
  return op;
}

Op add_op(const Labeled& lhs, double alpha, const Labeled& rhs) {
  Op op;
  op.kind      = Op::Add;
  op.lhs       = lhs;
  op.a         = rhs;
  op.alpha     = alpha;
  op.is_assign = 0;
  return op;
}

Op mult_op(const Labeled& lhs, double alpha, const Labeled& a, const Labeled& b) {
  Op op;
  op.kind  = Op::Mult;
  op.lhs   = lhs;
  op.a     = a;
  op.b     = b;
  op.alpha = alpha;
  return op;
}

} // namespace

// Adjoint label rule: every label of an operand must reach the other operand or the
// output, since its gradient is a contraction of those two (a label summed inside
// one operand alone would need a broadcast output).
void check_adjoint_labels(const Labeled& y, const Labeled& a, const Labeled& b) {
  for(int l: a.labels)
    if(!contains(y.labels, l) && !contains(b.labels, l))
      fail(TB_ERR_NOT_IMPLEMENTED, "adjoint of a contraction with a label summed inside the first operand alone");
  for(int l: b.labels)
    if(!contains(y.labels, l) && !contains(a.labels, l))
      fail(TB_ERR_NOT_IMPLEMENTED, "adjoint of a contraction with a label summed inside the second operand alone");
  for(int l: y.labels)
    if(!contains(a.labels, l) && !contains(b.labels, l)) fail(TB_ERR_INVALID, "output label in neither operand");
}

struct TapeNode {
  enum Kind { Contract, Dot } kind;
  Labeled y, a, b; // Dot: a = p, b = q
  double  alpha = 1.0;
};

struct Tape {
  std::shared_ptr<Ctx>                       ctx;
  Sched                                      sched;
  int64_t                                    budget = 0;
  std::vector<TapeNode>                      nodes;
  std::map<Tensor*, Tensor*>                 leaf_grad; // leaf -> its gradient (null: none)
  std::map<Tensor*, int>                     producer;  // Contract output -> node index
  std::set<Tensor*>                          dropped;
  std::map<Tensor*, std::unique_ptr<Tensor>> igrad; // gradients of Contract outputs
  int64_t                                    kept_bytes = 0, recomputed = 0;
  double                                     objective  = 0.0;

  void run_now() {
    sched.execute(false);
    TB_CUDA(cudaStreamSynchronize(ctx->stream));
  }

  void forward_contract(const TapeNode& n) {
    sched.ops.push_back(set_zero(n.y));
    sched.ops.push_back(mult_op(n.y, n.alpha, n.a, n.b));
    run_now();
  }

  // alpha * sum p * q with q's modes matched to p's by label
  double dot(double alpha, const Labeled& p, const Labeled& q) {
    p.t->require_allocated();
    q.t->require_allocated();
    if(p.labels == q.labels && same_layout(*p.t, *q.t))
      return alpha * reduce_dot(p.t->data, q.t->data, p.t->nelems, ctx->stream);
    auto tmp = clone_structure(*p.t, ctx); // q in p's layout
    sched.ops.push_back(set_zero(relabel(p, tmp.get())));
    sched.ops.push_back(add_op(relabel(p, tmp.get()), 1.0, q));
    run_now();
    const double s = reduce_dot(p.t->data, tmp->data, p.t->nelems, ctx->stream);
    ctx->arena->deallocate(tmp->data);
    tmp->data = nullptr;
    return alpha * s;
  }

  // value of t available (recomputing a dropped Contract output and its inputs)
  void ensure_value(Tensor* t) {
    if(!dropped.count(t)) return;
    const TapeNode& n = nodes[producer.at(t)];
    ensure_value(n.a.t);
    ensure_value(n.b.t);
    t->data = arena_alloc(ctx, t->nelems);
    t->ctx  = ctx;
    forward_contract(n);
    dropped.erase(t);
    recomputed++;
  }

  // gradient tensor of t: the caller's for a leaf, a zeroed clone for a Contract
  // output, null for a constant
  Tensor* grad_of(Tensor* t, bool create) {
    auto l = leaf_grad.find(t);
    if(l != leaf_grad.end()) return l->second;
    if(!producer.count(t)) return nullptr;
    auto g = igrad.find(t);
    if(g != igrad.end()) return g->second.get();
    if(!create) return nullptr;
    auto gt = clone_structure(*t, ctx);
    launch_fill(gt->data, gt->nelems, 0.0, 1, ctx->stream);
    Tensor* raw = gt.get();
    igrad[t]    = std::move(gt);
    return raw;
  }

  void backward() {
    // checkpoint decision, in recording order
    kept_bytes = 0;
    for(const auto& n: nodes) {
      if(n.kind != TapeNode::Contract || dropped.count(n.y.t)) continue;
      const int64_t bytes = (int64_t) sizeof(double) * n.y.t->nelems;
      if(kept_bytes + bytes <= budget) kept_bytes += bytes;
      else {
        ctx->arena->deallocate(n.y.t->data);
        n.y.t->data = nullptr;
        dropped.insert(n.y.t);
      }
    }
    for(auto it = nodes.rbegin(); it != nodes.rend(); ++it) {
      const TapeNode& n = *it;
      if(n.kind == TapeNode::Dot) {
        const Labeled &p = n.a, &q = n.b;
        if(Tensor* gp = grad_of(p.t, true)) {
          ensure_value(q.t);
          sched.ops.push_back(add_op(relabel(p, gp), n.alpha, q));
          run_now();
        }
        if(Tensor* gq = grad_of(q.t, true)) {
          ensure_value(p.t);
          sched.ops.push_back(add_op(relabel(q, gq), n.alpha, p));
          run_now();
        }
      }
      else {
        Tensor* gy = grad_of(n.y.t, false);
        if(!gy) continue; // the output does not reach the objective
        const Labeled dy = relabel(n.y, gy);
        if(Tensor* ga = grad_of(n.a.t, true)) {
          ensure_value(n.b.t);
          sched.ops.push_back(mult_op(relabel(n.a, ga), n.alpha, dy, n.b));
          run_now();
        }
        if(Tensor* gb = grad_of(n.b.t, true)) {
          ensure_value(n.a.t);
          sched.ops.push_back(mult_op(relabel(n.b, gb), n.alpha, n.a, dy));
          run_now();
        }
      }
    }
  }

  void reset() {
    for(auto& g: igrad)
      if(g.second->data) {
        ctx->arena->deallocate(g.second->data);
        g.second->data = nullptr;
      }
    igrad.clear();
    for(Tensor* t: dropped) { // freed outputs get their storage back
      t->data = arena_alloc(ctx, t->nelems);
      t->ctx  = ctx;
    }
    dropped.clear();
    nodes.clear();
    producer.clear();
    objective  = 0.0;
    kept_bytes = 0;
    recomputed = 0;
  }
};

} // namespace tb

struct tb_tape_s {
  std::unique_ptr<tb::Tape> p;
};

using namespace tb;

extern "C" {

int tb_tape_create(tb_ctx ctx, int64_t budget_bytes, tb_tape* out) {
  TB_API_BEGIN
  TB_EXPECTS(ctx != nullptr && out != nullptr, "ctx and out must be non-null");
  TB_EXPECTS(budget_bytes >= 0, "negative memory budget");
  auto t       = std::make_unique<Tape>();
  t->ctx       = ctx->p;
  t->sched.ctx = ctx->p;
  t->budget    = budget_bytes;
  auto* h      = new tb_tape_s();
  h->p         = std::move(t);
  *out         = h;
  TB_API_END
}

int tb_tape_destroy(tb_tape t) {
  if(t == nullptr) return TB_OK;
  try {
    t->p->reset();
  } catch(...) {
  }
  delete t;
  return TB_OK;
}

int tb_tape_leaf(tb_tape t, tb_tensor x, tb_tensor grad) {
  TB_API_BEGIN
  TB_EXPECTS(t != nullptr && x != nullptr, "tape and tensor must be non-null");
  Tensor* xt = x->p.get();
  TB_EXPECTS(!t->p->producer.count(xt), "a recorded Contract output cannot become a leaf");
  if(grad) {
    TB_EXPECTS(same_layout(*xt, *grad->p), "gradient tensor must have the leaf's spaces and spin mask");
    grad->p->require_allocated();
  }
  t->p->leaf_grad[xt] = grad ? grad->p.get() : nullptr;
  TB_API_END
}

int tb_tape_contract(tb_tape t, tb_labeled y, double alpha, tb_labeled a, tb_labeled b) {
  TB_API_BEGIN
  TB_EXPECTS(t != nullptr, "tape must be non-null");
  TapeNode n;
  n.kind  = TapeNode::Contract;
  n.y     = labeled_from_c(y);
  n.a     = labeled_from_c(a);
  n.b     = labeled_from_c(b);
  n.alpha = alpha;
  TB_EXPECTS(!t->p->leaf_grad.count(n.y.t) && !t->p->producer.count(n.y.t),
             "a Contract output must be a fresh tensor (not a leaf, not written before on this tape)");
  TB_EXPECTS(n.y.t != n.a.t && n.y.t != n.b.t, "a Contract output cannot be one of its operands");
  TB_EXPECTS(full_spaces(n.y), "a Contract output must be labelled over its full spaces");
  check_adjoint_labels(n.y, n.a, n.b);
  n.y.t->require_allocated();
  t->p->forward_contract(n);
  t->p->producer[n.y.t] = (int) t->p->nodes.size();
  t->p->nodes.push_back(n);
  TB_API_END
}

int tb_tape_dot(tb_tape t, double alpha, tb_labeled p, tb_labeled q, double* value) {
  TB_API_BEGIN
  TB_EXPECTS(t != nullptr, "tape must be non-null");
  TapeNode n;
  n.kind  = TapeNode::Dot;
  n.a     = labeled_from_c(p);
  n.b     = labeled_from_c(q);
  n.alpha = alpha;
  TB_EXPECTS(full_spaces(n.a) && full_spaces(n.b), "Dot operands must be labelled over their full spaces");
  TB_EXPECTS(n.a.labels.size() == n.b.labels.size(), "Dot operands need the same labels");
  for(int l: n.a.labels) TB_EXPECTS(contains(n.b.labels, l), "Dot operands need the same labels");
  const double s = t->p->dot(alpha, n.a, n.b);
  t->p->objective += s;
  t->p->nodes.push_back(n);
  if(value) *value = s;
  TB_API_END
}

int tb_tape_backward(tb_tape t) {
  TB_API_BEGIN
  TB_EXPECTS(t != nullptr, "tape must be non-null");
  t->p->backward();
  TB_API_END
}

int tb_tape_info(tb_tape t, int64_t* nnodes, double* objective, int64_t* kept_bytes, int64_t* recomputed) {
  TB_API_BEGIN
  TB_EXPECTS(t != nullptr, "tape must be non-null");
  if(nnodes) *nnodes = (int64_t) t->p->nodes.size();
  if(objective) *objective = t->p->objective;
  if(kept_bytes) *kept_bytes = t->p->kept_bytes;
  if(recomputed) *recomputed = t->p->recomputed;
  TB_API_END
}

int tb_tape_reset(tb_tape t) {
  TB_API_BEGIN
  TB_EXPECTS(t != nullptr, "tape must be non-null");
  t->p->reset();
  TB_API_END
}

} // extern "C"
