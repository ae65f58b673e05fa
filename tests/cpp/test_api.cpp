// C++ API tests, written the way TAMM's own doctest drivers are (tests/tamm/Test_Ops.cpp,
// Test_Mult_Ops.cpp): constant-filled tensors and known answers, plus a random-input
// contraction checked against host loops.  Built and run by tests/test_cpp_api.py.
#include "tamm_b200/tamm.hpp"

#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

using namespace tamm;

#define REQUIRE(cond)                                                            \
  do {                                                                           \
    if(!(cond)) {                                                                \
      std::fprintf(stderr, "FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond);     \
      return 1;                                                                  \
    }                                                                            \
  } while(0)

static bool check_value(const Tensor<double>& t, double v) {
  for(double x: t.read())
    if(std::fabs(x - v) > 1e-10) return false;
  return true;
}

// Test_Mult_Ops.cpp:176-204: N = 50 tiled 20 (tiles 20, 20, 10), |C| = 2.625e8.
static int test_4d_mult_norm(ExecutionContext& ec) {
  TiledIndexSpace tis1{IndexSpace{range(50)}, 20};
  REQUIRE(tis1.num_tiles() == 3 && tis1.tile_size(2) == 10);
  auto [i, j, k, l, m, o] = tis1.labels<6>("all");
  Tensor<double> A{i, j, m, o}, B{m, o, k, l}, C{i, j, k, l};
  Scheduler      sch{ec};
  sch.allocate(A, B, C);
  sch(A() = 21.0)(B() = 2.0)(C() = 0.0).execute();
  sch(C(j, i, k, l) += A(i, j, m, o) * B(m, o, k, l)).execute(ExecutionHW::GPU);
  REQUIRE(std::fabs(norm(C) - 2.625e8) <= 1e-9 * 2.625e8);
  sch.deallocate(A, B, C);
  return 0;
}

// Test_Ops.cpp:1396-1555: 3-D / 4-D mults with batch (Hadamard) labels, tile 1.
static int test_3d_4d_mult_ops(ExecutionContext& ec) {
  IndexSpace      IS{range(0, 10), {{"nr1", {range(0, 5)}}, {"nr2", {range(5, 10)}}}};
  TiledIndexSpace TIS{IS, 1};
  auto [i, j, k, l, m] = TIS.labels<5>("all");
  Scheduler sch{ec};
  {
    Tensor<double> T1{TIS, TIS, TIS}, T2{TIS, TIS, TIS}, T3{TIS, TIS, TIS};
    sch.allocate(T1, T2, T3);
    sch(T1() = 2)(T2() = 3)(T3() = 4)(T1(i, j, k) += 1.7 * T2(j, l, i) * T3(l, i, k)).execute();
    REQUIRE(check_value(T1, 2 + 1.7 * 3 * 4 * 10));
  }
  {
    Tensor<double> T1{TIS, TIS, TIS}, T2{TIS, TIS}, T3{TIS};
    sch.allocate(T1, T2, T3);
    sch(T1() = 2)(T2() = 3)(T3() = 4)(T1(i, j, k) += 1.7 * T2(i, j) * T3(k)).execute();
    REQUIRE(check_value(T1, 2 + 1.7 * 3 * 4));
  }
  {
    Tensor<double> T1{TIS, TIS, TIS}, T2{TIS, TIS, TIS}, T3{};
    sch.allocate(T1, T2, T3);
    sch(T1() = 2)(T2() = 3)(T3() = 4)(T1() += 6.9 * T2() * T3()).execute();
    REQUIRE(check_value(T1, 2 + 6.9 * 3 * 4));
  }
  {
    Tensor<double> T1{TIS, TIS, TIS, TIS}, T2{TIS, TIS, TIS, TIS}, T3{TIS, TIS, TIS, TIS};
    sch.allocate(T1, T2, T3);
    sch(T1() = 2)(T2() = 3)(T3() = 4)(T1(i, j, k, l) += 1.7 * T2(j, l, k, m) * T3(l, i, k, m)).execute();
    REQUIRE(check_value(T1, 2 + 1.7 * 3 * 4 * 10));
  }
  return 0;
}

// Test_TiledIndexSpace.cpp:308-328: tiles split at spin boundaries.
static int test_spin_tiling() {
  IndexSpace is_att{range(0, 20),
                    {{"occ", {range(0, 10)}}, {"virt", {range(10, 20)}}},
                    {{Spin{2}, {range(0, 5), range(10, 15)}}, {Spin{1}, {range(5, 10), range(15, 20)}}}};
  std::vector<Tile> tilesizes{3, 2, 3, 2, 3, 2, 3, 2};
  TiledIndexSpace   tis_att{is_att, 3};
  TiledIndexSpace   tis_att2{is_att, tilesizes};
  REQUIRE(tis_att.num_tiles() == 8 && tis_att2.num_tiles() == 8);
  for(int t = 0; t < 8; t++) REQUIRE(tis_att.tile_size(t) == tilesizes[t] && tis_att2.tile_size(t) == tilesizes[t]);
  return 0;
}

// Random-input contraction with string labels against host loops, FP64 and split-INT8.
static int test_random_contraction(ExecutionContext& ec, Precision p, double tol) {
  TiledIndexSpace Vt{IndexSpace{range(12)}, 5}, Ot{IndexSpace{range(6)}, 4};
  Tensor<double>  A{Vt, Vt, Ot, Ot}, B{Vt, Vt, Ot, Ot}, C{Vt, Vt, Ot, Ot};
  Scheduler       sch{ec};
  sch.allocate(A, B, C);
  std::mt19937_64                        g(7);
  std::uniform_real_distribution<double> U(-1, 1);
  // dense tensors: the packed store is the row-major order of the tile blocks
  std::vector<double> a(A.size()), b(B.size());
  for(auto& x: a) x = U(g);
  for(auto& x: b) x = U(g);
  A.write(a);
  B.write(b);
  ec.set_precision(p, 1e-11);
  sch(C("a,b,i,j") = 0.0)(C("a,b,i,j") += A("a,c,i,k") * B("c,b,k,j")).execute(ExecutionHW::GPU);
  ec.set_precision(Precision::FP64);
  // host reference, element by element through block get()
  auto dense = [](const Tensor<double>& T, const TiledIndexSpace& s0, const TiledIndexSpace& s1,
                  const TiledIndexSpace& s2, const TiledIndexSpace& s3) {
    std::vector<int64_t> z0 = s0.tile_sizes(), z1 = s1.tile_sizes(), z2 = s2.tile_sizes(), z3 = s3.tile_sizes();
    int64_t              n0 = 0, n1 = 0, n2 = 0, n3 = 0;
    for(auto x: z0) n0 += x;
    for(auto x: z1) n1 += x;
    for(auto x: z2) n2 += x;
    for(auto x: z3) n3 += x;
    std::vector<double> out(n0 * n1 * n2 * n3);
    int64_t             o0 = 0;
    for(int64_t t0 = 0; t0 < (int64_t) z0.size(); o0 += z0[t0++]) {
      int64_t o1 = 0;
      for(int64_t t1 = 0; t1 < (int64_t) z1.size(); o1 += z1[t1++]) {
        int64_t o2 = 0;
        for(int64_t t2 = 0; t2 < (int64_t) z2.size(); o2 += z2[t2++]) {
          int64_t o3 = 0;
          for(int64_t t3 = 0; t3 < (int64_t) z3.size(); o3 += z3[t3++]) {
            auto    blk = T.get({t0, t1, t2, t3});
            int64_t q   = 0;
            for(int64_t x0 = 0; x0 < z0[t0]; x0++)
              for(int64_t x1 = 0; x1 < z1[t1]; x1++)
                for(int64_t x2 = 0; x2 < z2[t2]; x2++)
                  for(int64_t x3 = 0; x3 < z3[t3]; x3++)
                    out[(((o0 + x0) * n1 + o1 + x1) * n2 + o2 + x2) * n3 + o3 + x3] = blk[q++];
          }
        }
      }
    }
    return out;
  };
  auto da = dense(A, Vt, Vt, Ot, Ot), db = dense(B, Vt, Vt, Ot, Ot), dc = dense(C, Vt, Vt, Ot, Ot);
  double maxerr = 0, maxref = 0;
  for(int ia = 0; ia < 12; ia++)
    for(int ib = 0; ib < 12; ib++)
      for(int ii = 0; ii < 6; ii++)
        for(int ij = 0; ij < 6; ij++) {
          double s = 0;
          for(int ic = 0; ic < 12; ic++)
            for(int ik = 0; ik < 6; ik++)
              s += da[((ia * 12 + ic) * 6 + ii) * 6 + ik] * db[((ic * 12 + ib) * 6 + ik) * 6 + ij];
          maxerr = std::fmax(maxerr, std::fabs(s - dc[((ia * 12 + ib) * 6 + ii) * 6 + ij]));
          maxref = std::fmax(maxref, std::fabs(s));
        }
  REQUIRE(maxerr <= tol * maxref);
  return 0;
}

// Dense host copy of a 2-mode tensor (no spin) through block get().
static std::vector<double> dense2(const Tensor<double>& T, const TiledIndexSpace& s0, const TiledIndexSpace& s1) {
  std::vector<int64_t> z0 = s0.tile_sizes(), z1 = s1.tile_sizes();
  int64_t              n0 = 0, n1 = 0;
  for(auto x: z0) n0 += x;
  for(auto x: z1) n1 += x;
  std::vector<double> out(n0 * n1);
  int64_t             o0 = 0;
  for(int64_t t0 = 0; t0 < (int64_t) z0.size(); o0 += z0[t0++]) {
    int64_t o1 = 0;
    for(int64_t t1 = 0; t1 < (int64_t) z1.size(); o1 += z1[t1++]) {
      auto    blk = T.get({t0, t1});
      int64_t q   = 0;
      for(int64_t x0 = 0; x0 < z0[t0]; x0++)
        for(int64_t x1 = 0; x1 < z1[t1]; x1++) out[(o0 + x0) * n1 + o1 + x1] = blk[q++];
    }
  }
  return out;
}

// Tape: E(t) = sum w(i,a) t(a,i) + 1/2 sum t(a,i) X(a,i), X = M(a,b) t(b,i);
// dE/dt(a,i) = w(i,a) + 1/2 X(a,i) + 1/2 sum_b M(b,a) t(b,i), against host loops,
// with the intermediate kept and with it recomputed (zero budget).
static int test_tape_gradient(ExecutionContext& ec, int64_t budget) {
  TiledIndexSpace Vt{IndexSpace{range(12)}, 5}, Ot{IndexSpace{range(6)}, 4};
  auto [a, b] = Vt.labels<2>("all");
  auto [i]    = Ot.labels<1>("all");
  Tensor<double> M{Vt, Vt}, t{Vt, Ot}, w{Ot, Vt}, X{Vt, Ot}, g{Vt, Ot};
  Scheduler      sch{ec};
  sch.allocate(M, t, w, X, g);
  std::mt19937_64                        gen(3);
  std::uniform_real_distribution<double> U(-1, 1);
  for(auto* T: {&M, &t, &w}) {
    std::vector<double> v(T->size());
    for(auto& x: v) x = U(gen);
    T->write(v);
  }
  sch(g() = 0.0).execute();
  Tape tape{ec, budget};
  tape.leaf(t, g);
  tape.contract(X(a, i), M(a, b) * t(b, i));
  const double E = tape.dot(w(i, a), t(a, i)) + tape.dot(t(a, i), X(a, i), 0.5);
  tape.backward();
  REQUIRE(tape.recomputed() == (budget == 0 ? 1 : 0));
  auto dm = dense2(M, Vt, Vt), dt = dense2(t, Vt, Ot), dw = dense2(w, Ot, Vt), dg = dense2(g, Vt, Ot);
  double e = 0, maxerr = 0, maxg = 0;
  for(int ia = 0; ia < 12; ia++)
    for(int ii = 0; ii < 6; ii++) {
      double x = 0, y = 0;
      for(int ib = 0; ib < 12; ib++) {
        x += dm[ia * 12 + ib] * dt[ib * 6 + ii];
        y += dm[ib * 12 + ia] * dt[ib * 6 + ii];
      }
      e += dw[ii * 12 + ia] * dt[ia * 6 + ii] + 0.5 * dt[ia * 6 + ii] * x;
      const double want = dw[ii * 12 + ia] + 0.5 * x + 0.5 * y;
      maxerr            = std::fmax(maxerr, std::fabs(want - dg[ia * 6 + ii]));
      maxg              = std::fmax(maxg, std::fabs(want));
    }
  REQUIRE(std::fabs(E - e) <= 1e-12 * std::fabs(e));
  REQUIRE(maxerr <= 1e-12 * maxg);
  return 0;
}

int main() {
  ExecutionContext ec{0, int64_t(2) << 30};
  int              rc = 0;
  rc |= test_spin_tiling();
  rc |= test_4d_mult_norm(ec);
  rc |= test_3d_4d_mult_ops(ec);
  rc |= test_random_contraction(ec, Precision::FP64, 1e-12);
  rc |= test_random_contraction(ec, Precision::INT8, 1e-11);
  rc |= test_tape_gradient(ec, INT64_MAX);
  rc |= test_tape_gradient(ec, 0);
  if(rc == 0) std::printf("ALL PASSED\n");
  return rc;
}
