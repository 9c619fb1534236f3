// Checks of the hand-written per-particle reverse (pdp3_b200/csrc/
// adjoint_particle.cuh) in double precision on the host:
//
// 1. pathwise: for random particles, fields and output adjoints, the reverse
//    equals central finite differences of sum(adjoint x output) with respect
//    to the particle's offsets, momentum, weight and gathered field values,
//    for steps that cross cell faces, reflect at the walls, or remove a bunch
//    particle (differences that change the branch taken are skipped);
// 2. mean field: for particles spread uniformly over whole cells, the
//    pathwise gather derivative plus radial_jump() equals the central
//    difference of the particles' mean gathered value under a common radial
//    shift, which includes the weights' jumps at faces and cell middles
//    (also for windows that start or end in the half of a wall cell that the
//    walls leave to particles, with the wall-cell share);
// 3. the same for the momentum jumps of the wall reflections (wall_jumps()).
// Prints one line per check and exits non-zero on failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "adjoint_particle.cuh"

using namespace pdp3g::adj;
typedef double T;

static std::mt19937_64 rng(1);
static double U(double a, double b) { return std::uniform_real_distribution<double>(a, b)(rng); }

struct In {
  int i, k;
  T a, b, u[3], w, fe[3][4], fh[3][4];
};
struct LamOut {
  T an, bn, u[3], jphi[4], piece[3][4];
};

static T objective(const Consts<T> &C, const In &in, const LamOut &L, Tape<T> *keep) {
  Tape<T> tp;
  tp.i = in.i;
  tp.k = in.k;
  tp.a = in.a;
  tp.b = in.b;
  tp.w = in.w;
  for (int c = 0; c < 3; c++) {
    tp.u[c] = in.u[c];
    for (int n = 0; n < 4; n++) {
      tp.fe[c][n] = in.fe[c][n];
      tp.fh[c][n] = in.fh[c][n];
    }
  }
  forward(C, tp);
  if (keep) *keep = tp;
  T s = 0;
  if (tp.alive_now) s += L.an * tp.A + L.bn * tp.B;  // A, B: the outputs up to a cell shift
  for (int c = 0; c < 3; c++) s += L.u[c] * tp.uout[c];
  const T jp[4] = {tp.pref * (1 - tp.g1) * tp.wa, tp.pref * (1 - tp.g1) * tp.wb,
                   tp.pref * tp.g1 * tp.wa, tp.pref * tp.g1 * tp.wb};
  for (int n = 0; n < 4; n++) s += L.jphi[n] * jp[n];
  if (tp.path_ok)
    for (int p = 0; p <= tp.np; p++) {
      T o[4];
      piece_outputs(C, tp, p, o);
      for (int n = 0; n < 4; n++) s += L.piece[p][n] * o[n];
    }
  return s;
}

static bool same_branch(const Tape<T> &x, const Tape<T> &y) {
  return x.in == y.in && x.kn == y.kn && x.i1 == y.i1 && x.k1 == y.k1 && x.np == y.np &&
         x.ir_h == y.ir_h && x.kz_h == y.kz_h && x.sr == y.sr && x.sz == y.sz &&
         x.alive_now == y.alive_now && (x.np == 0 || x.kind0 == y.kind0);
}

static int pathwise() {
  Consts<T> C;
  C.ke = 0.3; C.kb = 0.7; C.cr = 0.11; C.cz = 0.13; C.kphi = 1.3; C.kz = 0.9; C.kr = 1.1;
  C.nr = 40; C.nz = 60; C.bunch = 0; C.face = 0;
  double worst = 0;
  int tested = 0, crossing = 0, reflected = 0, removed = 0;
  for (int trial = 0; trial < 4000; trial++) {
    In in;
    in.i = (trial % 5 == 0) ? 0 : 1 + (int)(rng() % 30);
    in.k = 1 + (int)(rng() % 50);
    if (trial % 7 == 1) { in.i = C.nr - 2; in.k = C.nz - 2; }  // outer walls
    if (trial % 7 == 2) { in.i = 0; in.k = 0; }                // axis and z = 0 wall
    C.bunch = (trial % 11 == 3);
    in.a = U(0.02, 0.98);
    in.b = U(0.02, 0.98);
    for (int c = 0; c < 3; c++) {
      in.u[c] = U(-0.8, 0.8);
      for (int n = 0; n < 4; n++) { in.fe[c][n] = U(-1, 1); in.fh[c][n] = U(-1, 1); }
    }
    if (trial % 3 == 0 || trial % 7 == 1 || trial % 7 == 2) { in.u[0] *= 6; in.u[2] *= 6; }
    if (trial % 7 == 1) {
      in.a = U(0.3, 0.98); in.b = U(0.3, 0.98);
      in.u[0] = std::fabs(in.u[0]) + 1.5; in.u[2] = std::fabs(in.u[2]) + 1.5;
    }
    if (trial % 7 == 2) {
      in.a = U(0.5, 0.9); in.b = U(0.5, 0.9);
      in.u[0] = -std::fabs(in.u[0]) - 2; in.u[2] = -std::fabs(in.u[2]) - 2;
    }
    in.w = U(0.5, 2);
    LamOut L;
    L.an = U(-1, 1); L.bn = U(-1, 1);
    for (int c = 0; c < 3; c++) L.u[c] = U(-1, 1);
    for (int n = 0; n < 4; n++) L.jphi[n] = U(-1, 1);
    for (int p = 0; p < 3; p++)
      for (int n = 0; n < 4; n++) L.piece[p][n] = U(-1, 1);
    Tape<T> tp;
    objective(C, in, L, &tp);
    T la, lb, lu[3], lw, lfe[3][4], lfh[3][4];
    reverse(C, tp, L.an, L.bn, L.u, L.jphi, L.piece, la, lb, lu, lw, lfe, lfh);
    auto fd = [&](auto setter) {
      const double h = 1e-6;
      In p = in, m = in;
      setter(p, h);
      setter(m, -h);
      Tape<T> tpp, tpm;
      const T fp = objective(C, p, L, &tpp), fm = objective(C, m, L, &tpm);
      if (!same_branch(tpp, tp) || !same_branch(tpm, tp)) return (double)NAN;
      return (double)((fp - fm) / (2 * h));
    };
    double g[12];
    const double ad[12] = {la, lb, lu[0], lu[1], lu[2], lw, lfe[0][1], lfe[2][2],
                           lfh[1][3], lfh[0][0], lfe[1][0], lfh[2][1]};
    g[0] = fd([](In &x, double h) { x.a += h; });
    g[1] = fd([](In &x, double h) { x.b += h; });
    g[2] = fd([](In &x, double h) { x.u[0] += h; });
    g[3] = fd([](In &x, double h) { x.u[1] += h; });
    g[4] = fd([](In &x, double h) { x.u[2] += h; });
    g[5] = fd([](In &x, double h) { x.w += h; });
    g[6] = fd([](In &x, double h) { x.fe[0][1] += h; });
    g[7] = fd([](In &x, double h) { x.fe[2][2] += h; });
    g[8] = fd([](In &x, double h) { x.fh[1][3] += h; });
    g[9] = fd([](In &x, double h) { x.fh[0][0] += h; });
    g[10] = fd([](In &x, double h) { x.fe[1][0] += h; });
    g[11] = fd([](In &x, double h) { x.fh[2][1] += h; });
    if (tp.np > 0) crossing++;
    if (tp.sr < 0 || tp.sz < 0) reflected++;
    if (!tp.alive_now) removed++;
    for (int j = 0; j < 12; j++) {
      if (std::isnan(g[j])) continue;
      const double e = std::fabs(g[j] - ad[j]) / std::fmax(1.0, std::fabs(g[j]));
      if (e > worst) worst = e;
      tested++;
    }
  }
  printf("pathwise: %d derivatives (%d steps crossing faces, %d reflected, %d removed), "
         "worst rel err %.3g\n", tested, crossing, reflected, removed, worst);
  return (worst < 1e-6 && tested > 40000 && crossing > 500 && reflected > 500 && removed > 20) ? 0 : 1;
}

// gathered value of a component at radial coordinate x (cells), fixed z weights
static T gather_at(T x, const T *F0, const T *F1, T b, bool rh, bool zh, bool wall_cells, int nr,
                   T face_h, T *dG, T *jump) {
  Tape<T> tp;
  tp.i = (int)std::ceil(x) - 1;
  tp.a = x - tp.i;
  tp.k = 3;
  tp.b = b;
  gather_weights(tp);
  const int ir = rh ? tp.ir_h : tp.i;
  const T f[4] = {F0[ir], F0[ir + 1], F1[ir], F1[ir + 1]};
  const T *wr = rh ? tp.wrh : tp.wrn, *dwr = rh ? tp.dwrh : tp.dwrn;
  const T *wz = zh ? tp.wzh : tp.wzn;
  if (dG) *dG = wz[0] * (f[0] * dwr[0] + f[1] * dwr[1]) + wz[1] * (f[2] * dwr[0] + f[3] * dwr[1]);
  if (jump)
    *jump = radial_jump(tp, f[0], f[1], f[2], f[3], wz[0], wz[1], rh, wall_cells, nr, face_h);
  return wz[0] * (f[0] * wr[0] + f[1] * wr[1]) + wz[1] * (f[2] * wr[0] + f[3] * wr[1]);
}

// Windows of whole cells; with wall_cells, windows that start in the axis
// cell at r = dr/2 or end in the last cell (nr - 2) at r = r_max - dr/2, the
// parts of those cells that the walls leave to particles.  Each window is
// checked with the uniform-density shares (face_h = 0) and with box-kernel
// shares of half-width 1/4 and 1/8 cell, which count the particles actually
// near each jump (the wall-cell flag then has no role).
static int mean_field() {
  double worst = 0;
  int cases = 0;
  for (int trial = 0; trial < 108; trial++) {
    const T face_h = trial < 36 ? 0.0 : (trial < 72 ? 0.25 : 0.125);
    T F0[64], F1[64];
    for (int j = 0; j < 64; j++) { F0[j] = U(-1, 1) + 2; F1[j] = U(-1, 1) + 2; }
    const bool rh = trial % 2, zh = (trial / 2) % 2;
    const int wall = trial % 36 < 24 ? 0 : 1 + trial % 3 % 2;  // 1: axis cell, 2: last cell
    int i0 = 1 + (int)(rng() % 20), i1 = i0 + 1 + (int)(rng() % 8);
    if (wall == 1) i0 = 0;
    const int nr = wall == 2 ? i1 + 1 : 64;  // with wall == 2 the window ends in cell nr - 2
    const T b = U(0.05, 0.95);
    // midpoint rule with a whole number of points per cell and shifts of a
    // whole number of point spacings: exactly that many points cross each
    // face, so the differences resolve the jumps without quadrature error.
    // The weights also have kinks at the faces, which make the central
    // difference O(h); Richardson extrapolation over h and 2h removes that.
    const int per_cell = 50000;
    const int q0 = wall == 1 ? per_cell / 2 : 0;
    const int q1 = per_cell * (i1 - i0) - (wall == 2 ? per_cell / 2 : 0);
    const int n = q1 - q0;
    const T h = 50.0 / per_cell;
    double mp = 0, mm = 0, mp2 = 0, mm2 = 0, est = 0;
    for (int q = q0; q < q1; q++) {
      const T x = i0 + (q + 0.5) / per_cell;
      T dG, jump;
      gather_at(x, F0, F1, b, rh, zh, wall != 0, nr, face_h, &dG, &jump);
      est += dG + jump;
      mp += gather_at(x + h, F0, F1, b, rh, zh, false, nr, 0, nullptr, nullptr);
      mm += gather_at(x - h, F0, F1, b, rh, zh, false, nr, 0, nullptr, nullptr);
      mp2 += gather_at(x + 2 * h, F0, F1, b, rh, zh, false, nr, 0, nullptr, nullptr);
      mm2 += gather_at(x - 2 * h, F0, F1, b, rh, zh, false, nr, 0, nullptr, nullptr);
    }
    const double d1 = (mp - mm) / (2 * h) / n, d2 = (mp2 - mm2) / (4 * h) / n;
    const double fd = 2 * d1 - d2, ad = est / n;
    // relative to |fd|, floored at 1e-2 (the field values are in [1, 3]): a
    // window whose jumps nearly cancel has an fd near 0, and the midpoint
    // rule's absolute error there (~5e-7) says nothing about the shares
    const double e = std::fabs(fd - ad) / std::fmax(std::fabs(fd), 1e-2);
    if (e > worst) worst = e;
    if (getenv("ADJ_VERBOSE"))
      printf("  rh %d zh %d wall %d face_h %.3f cells [%d,%d) fd %.6g est %.6g\n", rh, zh, wall,
             face_h, i0, i1, fd, ad);
    cases++;
  }
  printf("mean field: %d windows, worst rel err %.3g\n", cases, worst);
  return worst < 1e-4 ? 0 : 1;
}

// 3. wall reflections: with zero fields and adjoints on the end point and the
//    momentum only, S = sum(adjoint x output) is piecewise smooth in the start
//    offset a (b) with jumps where the end point meets a wall, so the mean of
//    the reverse's l_a (l_b) with the wall terms on over the part of the cell
//    that particles occupy ([1/2, 1) next to the axis and z = 0, [0, 1/2)
//    next to the outer walls, else [0, 1)) equals the difference quotient of S
//    over that part (to the midpoint rule's O(1/n) at the kinks; the jumps
//    are O(1) here).
static int wall_mean_field() {
  double worst = 0;
  int cases = 0, with_jump = 0;
  for (int trial = 0; trial < 60; trial++) {
    Consts<T> C;
    C.ke = 0.3; C.kb = 0.7; C.cz = 0.13; C.kphi = 1.3; C.kz = 0.9; C.kr = 1.1;
    C.nr = 40; C.nz = 60; C.face = 2;
    In in = {};
    const int kind = trial % 3;  // 0: axis and z = 0, 1: outer walls, 2: cell 1 and middle
    C.cr = trial % 6 == 3 ? 2.0 : 0.11;  // on the axis: the threshold at x < 0 too
    C.bunch = trial % 4 == 3 && kind != 1;  // a bunch particle is removed at the outer walls
    in.i = kind == 0 ? 0 : (kind == 1 ? C.nr - 2 : 1);
    in.k = kind == 0 ? 0 : (kind == 1 ? C.nz - 2 : 20);
    in.b = U(0.1, 0.9);
    in.a = U(0.1, 0.9);
    in.w = 1;
    const T sgn = kind == 1 ? 1 : -1;
    in.u[0] = sgn * U(1, 8);
    in.u[1] = U(-1, 1);
    in.u[2] = sgn * U(1, 8);
    if (C.cr > 1) {
      // velocity (-0.6, +-0.795, 0.02) c: the x < 0 threshold lies at a = 0.6
      const T v[3] = {-0.6, 0.795 * (trial % 4 == 3 ? 1 : -1), 0.02};
      const T g = 1 / std::sqrt(1 - v[0] * v[0] - v[1] * v[1] - v[2] * v[2]);
      for (int c = 0; c < 3; c++) in.u[c] = g * v[c];
    }
    LamOut L = {};
    L.an = U(-1, 1); L.bn = U(-1, 1);
    for (int c = 0; c < 3; c++) L.u[c] = U(-1, 1);
    for (int dir = 0; dir < 2; dir++) {
      const T lo_edge = kind == 0 ? 0.5 : 0, hi_edge = kind == 1 ? 0.5 : 1;
      const int n = 20000;
      double mean = 0;
      for (int q = 0; q < n; q++) {
        In x = in;
        (dir == 0 ? x.a : x.b) = lo_edge + (hi_edge - lo_edge) * (q + 0.5) / n;
        Tape<T> tp;
        objective(C, x, L, &tp);
        T la, lb, lu[3], lw, lfe[3][4], lfh[3][4];
        reverse(C, tp, L.an, L.bn, L.u, L.jphi, L.piece, la, lb, lu, lw, lfe, lfh);
        mean += (dir == 0 ? la : lb);
      }
      mean /= n;
      In lo = in, hi = in;
      (dir == 0 ? lo.a : lo.b) = lo_edge + 1e-13;
      (dir == 0 ? hi.a : hi.b) = hi_edge - 1e-13;
      Tape<T> tlo, thi;
      const double want =
          (objective(C, hi, L, &thi) - objective(C, lo, L, &tlo)) / (hi_edge - lo_edge);
      if (thi.sr != tlo.sr || thi.sz != tlo.sz) with_jump++;
      const double e = std::fabs(mean - want) / std::fmax(std::fabs(want), 1.0);
      if (e > worst) worst = e;
      if (getenv("ADJ_VERBOSE"))
        printf("  trial %d dir %d i %d k %d bunch %d: dS/d(offset) %.9g mean l %.9g\n", trial,
               dir, in.i, in.k, C.bunch, want, mean);
      cases++;
    }
  }
  printf("wall mean field: %d cells (%d with a reflection threshold), worst rel err %.3g\n",
         cases, with_jump, worst);
  return (worst < 1e-4 && with_jump > 30) ? 0 : 1;
}

int main() {
  const int a = pathwise();
  const int b = mean_field();
  const int c = wall_mean_field();
  return a | b | c;
}
