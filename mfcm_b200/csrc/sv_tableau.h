// sv_tableau.h -- the named Runge-Kutta tableaux, shared by every host path that launches the
// stage kernels (the solver, batches and the allocation-free timestep), so that all of them
// take their coefficients from one table.
#pragma once
#include <vector>

namespace svt {

// Butcher tableau in the reference's row layout: row i-1 holds (c_i, a_i1, ..., a_i,i-1) for
// stage i, the last row (0, b_1, ..., b_N).
struct Tableau {
  std::vector<std::vector<double>> a;
  int nsteps() const { return int(a.size()) - 1; }
  double A(int i, int j) const { return a[i - 1][j]; }
  double b(int i) const { return a[a.size() - 1][i]; }
  double c(int i) const { return a[i - 1][0]; }
};

// runge_kutta_named_coefficient_sets_ (src/TemporalScheme/RungeKutta.cpp:54-115), in its
// index order: euler, midpoint, heun2, ralston2, kutta3, heun3, wray3, ralston3, ssprk3,
// classic, ralston4, 3/8 rule
inline bool named_tableau(int id, Tableau& t) {
  switch (id) {
    case 0: t.a = {{0.0}, {0.0, 1.0}}; return true;
    case 1: t.a = {{0.0}, {0.5, 0.5}, {0.0, 0.0, 1.0}}; return true;
    case 2: t.a = {{0.0}, {1.0, 1.0}, {0.0, 0.5, 0.5}}; return true;
    case 3: t.a = {{0.0}, {2.0 / 3.0, 2.0 / 3.0}, {0.0, 0.25, 0.75}}; return true;
    case 4: t.a = {{0.0}, {0.5, 0.5}, {1.0, -1.0, 2.0}, {0.0, 1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0}}; return true;
    case 5: t.a = {{0.0}, {1.0 / 3.0, 1.0 / 3.0}, {2.0 / 3.0, 0.0, 2.0 / 3.0}, {0.0, 0.25, 0.0, 0.75}}; return true;
    case 6: t.a = {{0.0}, {8.0 / 15.0, 8.0 / 15.0}, {2.0 / 3.0, 0.25, 5.0 / 12.0}, {0.0, 0.25, 0.0, 0.75}}; return true;
    case 7: t.a = {{0.0}, {0.5, 0.5}, {0.75, 0.0, 0.75}, {0.0, 2.0 / 9.0, 1.0 / 3.0, 4.0 / 9.0}}; return true;
    case 8: t.a = {{0.0}, {1.0, 1.0}, {0.5, 0.25, 0.25}, {0.0, 1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0}}; return true;
    case 9:
      t.a = {{0.0}, {0.5, 0.5}, {0.5, 0.0, 0.5}, {1.0, 0.0, 0.0, 1.0}, {0.0, (1.0 / 6.0), (1.0 / 3.0), (1.0 / 3.0), (1.0 / 6.0)}};
      return true;
    case 10:
      t.a = {{0.0}, {0.4, 0.4}, {0.45573725, 0.29697761, 0.15875964}, {1.0, 0.21810040, -3.05096516, 3.83286476},
             {0.0, 0.17476028, -0.55148066, 1.20553560, 0.17118478}};
      return true;
    case 11:
      t.a = {{0.0}, {1.0 / 3.0, 1.0 / 3.0}, {2.0 / 3.0, -1.0 / 3.0, 1.0}, {1.0, 1.0, -1.0, 1.0},
             {0.0, 1.0 / 8.0, 3.0 / 8.0, 3.0 / 8.0, 1.0 / 8.0}};
      return true;
  }
  return false;
}

// Y_{s+1} depends on k_s alone (every earlier coefficient is zero): the stages can keep a
// running accumulator instead of storing the k's.
inline bool is_diagonal(const Tableau& t) {
  int N = t.nsteps();
  for (int s = 0; s + 1 < N; ++s)
    for (int j = 0; j < s; ++j)
      if (t.A(s + 2, j + 1) != 0.0) return false;
  return true;
}

// Per-stage launch coefficients of a tableau of at most 4 stages: c_s of each stage, the
// coefficients a(s+2, j+1) of Y_{s+1} (j <= s) and b_1..b_N, zero-filled.
struct StageCoefs {
  int N = 0;
  double c[4] = {}, a_next[4][4] = {}, b[4] = {};
};
inline bool stage_coefs(const Tableau& t, StageCoefs& k) {
  k = StageCoefs{};
  k.N = t.nsteps();
  if (k.N < 1 || k.N > 4) return false;
  for (int st = 0; st < k.N; ++st) {
    k.c[st] = t.c(st + 1);
    if (st < k.N - 1)
      for (int j = 0; j <= st; ++j) k.a_next[st][j] = t.A(st + 2, j + 1);
    k.b[st] = t.b(st + 1);
  }
  return true;
}

}  // namespace svt
