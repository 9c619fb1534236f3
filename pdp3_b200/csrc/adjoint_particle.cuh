// Hand-written reverse mode (vector-Jacobian product) of one particle's part
// of the FP32 cell-local step (particles_f32.cuh): gather, relativistic
// Boris, the two half moves with the rz rotation and the walls, the
// azimuthal deposition and the r-z deposition with its segment split.
//
// forward() recomputes the particle's step and records the intermediates in
// a Tape; reverse() takes the adjoints of the particle's outputs (position,
// momentum) and of the grid currents at the nodes it deposited into, and
// returns the adjoints of its inputs (offsets, momentum, weight) and of the
// field values it gathered.  Both are templates on the scalar type so the
// reverse can be checked against finite differences in double on the host;
// the GPU instantiates them with float, the precision of the forward.
// Branches (cell crossings, walls) are those the forward takes: the VJP is
// the derivative of the branch taken.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define PDP3_HD __host__ __device__ __forceinline__
// rare branches: out of line on the GPU, so that the particle loop keeps
// none of their code (arguments and results by value)
#define PDP3_COLD __host__ __device__ __noinline__
#else
#define PDP3_HD inline
#define PDP3_COLD inline
#endif


namespace pdp3g {
namespace adj {

template <typename T>
struct Consts {
  T ke, kb;     // Boris: charge dt / (2 mass c), mu0 charge dt / (2 mass)
  T cr, cz;     // c dt / (2 dr), c dt / (2 dz)
  T kphi, kz, kr;  // deposition prefactors per unit weight
  int nr, nz;   // grid nodes
  int bunch;    // 1: outer walls remove the particle
  T face_h = T(0);  // > 0: the gather jump terms from the particles within
                   // face_h (cells) of each jump, a box-kernel estimate of
                   // the density there; 0: density uniform inside each cell
  int face;     // bit 0: expected jump terms of the radial gather weights;
                // bit 1: expected jump terms of the wall reflections;
                // bit 2: the gather terms with the wall cells' particles in
                //        the half of the cell that the walls leave them
                // (PDP3G_ADJ_GATHER_JUMPS, _WALL_JUMPS, _WALL_CELLS)
};

template <typename T>
struct Tape {
  int i, k;
  T a, b, u[3], w;
  // gather
  int ir_h, kz_h;
  T wrh[2], wrn[2], wzh[2], wzn[2], dwrh[2], dwrn[2];
  T fe[3][4], fh[3][4];
  T e[3], h[3];
  // push
  T um[3], gi, tb[3], c2, wv[3], v2[3], up[3], inv_g, vel[3];
  // first half move and j_phi
  T dr_h, dy, dz_h, x, rr, b1;
  int i1, k1;
  T f1, g1, wa, wb, dwa, dwb, pref;
  // second half move, walls, rotation
  T sr, sz, ur_sign, uz_sign, x2, r2, A, B;
  bool alive_now;
  int in, kn;
  T an, bn, st, ct, uout[3];
  // r-z path: points Q0..Q(np+1) relative to the start cell (qa, qb),
  // piece p in cell (pci_p, pck_p), crossing p at parameter ts_p through an
  // r face (kind 0) or a z face (kind 1).  Scalars, not arrays, so that the
  // compiler keeps the whole tape in registers.
  int np, kind0, kind1, pci0, pci1, pci2, pck0, pck1, pck2;
  T ts0, ts1, qa0, qa1, qa2, qa3, qb0, qb1, qb2, qb3;
  bool path_ok;
  PDP3_HD T qa(int p) const { return p == 0 ? qa0 : (p == 1 ? qa1 : (p == 2 ? qa2 : qa3)); }
  PDP3_HD T qb(int p) const { return p == 0 ? qb0 : (p == 1 ? qb1 : (p == 2 ? qb2 : qb3)); }
  PDP3_HD int pci(int p) const { return p == 0 ? pci0 : (p == 1 ? pci1 : pci2); }
  PDP3_HD int pck(int p) const { return p == 0 ? pck0 : (p == 1 ? pck1 : pck2); }
  PDP3_HD T ts(int p) const { return p == 0 ? ts0 : ts1; }
  PDP3_HD int kind(int p) const { return p == 0 ? kind0 : kind1; }
};

template <typename T>
PDP3_HD T tmin(T x, T y) { return x < y ? x : y; }

// element p of a 3- or 4-entry tape array by selects (no run-time indexing)
template <typename T>
PDP3_HD T sel3(int p, T a0, T a1, T a2) { return p == 0 ? a0 : (p == 1 ? a1 : a2); }
template <typename T>
PDP3_HD T sel4(int p, T a0, T a1, T a2, T a3) {
  return p == 0 ? a0 : (p == 1 ? a1 : (p == 2 ? a2 : a3));
}

// ---------------------------------------------------------------- pieces

template <typename T>
struct EpsDeriv {
  T eps, deps;
};

// eps and its derivative for s^2 >= 0.01 (a radial move of a fifth of the
// radius or more in one piece: rare)
template <typename T>
PDP3_COLD EpsDeriv<T> eps_far(T s) {
  const T at = atanh(s);
  return EpsDeriv<T>{at / s - T(1), (T(1) / (T(1) - s * s) - at / s) / s};
}

// eps(s) = atanh(s)/s - 1 and its derivative
template <typename T>
PDP3_HD void eps_and_deriv(T s, T &eps, T &deps) {
  const T s2 = s * s;
  if (s2 < T(0.01)) {
    eps = s2 * (T(1) / 3 + s2 * (T(0.2) + s2 * (T(1) / 7 + s2 * (T(1) / 9))));
    deps = s * (T(2) / 3 + s2 * (T(0.8) + s2 * (T(6) / 7 + s2 * (T(8) / 9))));
  } else {
    const EpsDeriv<T> r = eps_far(s);
    eps = r.eps;
    deps = r.deps;
  }
}

// piece values (particles_f32.cuh piece_values) for cell column ci
template <typename T>
PDP3_HD void piece_fwd(int ci, T ao, T co, T an, T cn, T kz, T kr, T out[4]) {
  const T drho = an - ao, dzeta = cn - co, fi = T(ci), fm = T(0.5) * (ao + an);
  const T rho_m = fi + fm, beta = T(1) - co;
  if (ci >= 1) {
    T eps, deps;
    eps_and_deriv(T(0.5) * drho / rho_m, eps, deps);
    const T ii1 = fi * (fi + 1), h = T(0.5) * ii1;
    const T rho_o = fi + ao, rho_n = fi + an;
    out[0] = kz * dzeta * ((1 - fm) * (2 * fi + fm) + ii1 * eps) / rho_m / fi;
    out[1] = kz * dzeta * (fm * (2 * fi + 1 + fm) - ii1 * eps) / rho_m / (fi + 1);
    const T q1 = drho / (rho_o * rho_n), q2 = dzeta * drho / (2 * rho_n * rho_m);
    const T q3 = dzeta * eps / rho_m, pr = kr / (fi + T(0.5));
    out[2] = pr * (T(0.5) * drho * beta - T(0.25) * dzeta * drho + h * (q1 * beta - q2 - q3));
    out[3] = pr * (T(0.5) * drho * co + T(0.25) * dzeta * drho + h * (q1 * co + q2 + q3));
  } else {
    out[0] = 8 * kz * dzeta * (1 - fm);
    out[1] = kz * dzeta * (1 + fm);
    out[2] = 2 * kr * (T(0.5) * drho * beta - T(0.25) * dzeta * drho);
    out[3] = 2 * kr * (T(0.5) * drho * co + T(0.25) * dzeta * drho);
  }
}

// adjoint of piece_fwd: lo = adjoints of the 4 outputs; adds into the
// endpoint adjoints and returns the adjoint of the (kz, kr) scale (the
// outputs are linear in kz for j_z and in kr for j_r)
template <typename T>
PDP3_HD void piece_rev(int ci, T ao, T co, T an, T cn, T kz, T kr, const T lo[4], T &l_ao,
                       T &l_co, T &l_an, T &l_cn, T &l_kz, T &l_kr) {
  const T drho = an - ao, dzeta = cn - co, fi = T(ci), fm = T(0.5) * (ao + an);
  const T rho_m = fi + fm, beta = T(1) - co;
  T l_drho = 0, l_dzeta = 0, l_fm = 0, l_beta = 0, l_co_direct = 0;
  if (ci >= 1) {
    const T s = T(0.5) * drho / rho_m;
    T eps, deps;
    eps_and_deriv(s, eps, deps);
    const T ii1 = fi * (fi + 1), h = T(0.5) * ii1;
    const T rho_o = fi + ao, rho_n = fi + an;
    // out0 = kz dzeta N0 / (rho_m fi), N0 = (1-fm)(2fi+fm) + ii1 eps
    const T N0 = (1 - fm) * (2 * fi + fm) + ii1 * eps;
    const T N1 = fm * (2 * fi + 1 + fm) - ii1 * eps;
    const T o0 = kz * dzeta * N0 / rho_m / fi, o1 = kz * dzeta * N1 / rho_m / (fi + 1);
    T l_eps = 0, l_rho_m = 0;
    l_kz += lo[0] * o0 / kz + lo[1] * o1 / kz;
    {
      const T c0 = kz / (rho_m * fi), c1 = kz / (rho_m * (fi + 1));
      l_dzeta += lo[0] * c0 * N0 + lo[1] * c1 * N1;
      const T lN0 = lo[0] * c0 * dzeta, lN1 = lo[1] * c1 * dzeta;
      l_rho_m += -lo[0] * o0 / rho_m - lo[1] * o1 / rho_m;
      // dN0/dfm = -(2fi+fm) + (1-fm) ; dN1/dfm = 2fi+1+2fm
      l_fm += lN0 * (-(2 * fi + fm) + (1 - fm)) + lN1 * (2 * fi + 1 + 2 * fm);
      l_eps += lN0 * ii1 - lN1 * ii1;
    }
    // j_r
    const T pr = kr / (fi + T(0.5));
    const T q1 = drho / (rho_o * rho_n), q2 = dzeta * drho / (2 * rho_n * rho_m);
    const T q3 = dzeta * eps / rho_m;
    const T S2 = T(0.5) * drho * beta - T(0.25) * dzeta * drho + h * (q1 * beta - q2 - q3);
    const T S3 = T(0.5) * drho * co + T(0.25) * dzeta * drho + h * (q1 * co + q2 + q3);
    l_kr += (lo[2] * S2 + lo[3] * S3) / (fi + T(0.5));
    const T lS2 = lo[2] * pr, lS3 = lo[3] * pr;
    l_drho += lS2 * (T(0.5) * beta - T(0.25) * dzeta) + lS3 * (T(0.5) * co + T(0.25) * dzeta);
    l_dzeta += lS2 * (-T(0.25) * drho) + lS3 * (T(0.25) * drho);
    l_beta += lS2 * (T(0.5) * drho + h * q1);
    l_co_direct += lS3 * (T(0.5) * drho + h * q1);
    const T l_q1 = h * (lS2 * beta + lS3 * co);
    const T l_q2 = h * (-lS2 + lS3);
    const T l_q3 = h * (-lS2 + lS3);
    // q1 = drho / (rho_o rho_n)
    l_drho += l_q1 / (rho_o * rho_n);
    const T l_rho_o = -l_q1 * q1 / rho_o, l_rho_n1 = -l_q1 * q1 / rho_n;
    // q2 = dzeta drho / (2 rho_n rho_m)
    l_dzeta += l_q2 * drho / (2 * rho_n * rho_m);
    l_drho += l_q2 * dzeta / (2 * rho_n * rho_m);
    const T l_rho_n2 = -l_q2 * q2 / rho_n;
    l_rho_m += -l_q2 * q2 / rho_m;
    // q3 = dzeta eps / rho_m
    l_dzeta += l_q3 * eps / rho_m;
    l_eps += l_q3 * dzeta / rho_m;
    l_rho_m += -l_q3 * q3 / rho_m;
    // eps(s), s = drho / (2 rho_m)
    const T l_s = l_eps * deps;
    l_drho += l_s / (2 * rho_m);
    l_rho_m += -l_s * s / rho_m;
    // rho_m = fi + fm, rho_o = fi + ao, rho_n = fi + an
    l_fm += l_rho_m;
    l_ao += l_rho_o;
    l_an += l_rho_n1 + l_rho_n2;
  } else {
    const T o0 = 8 * kz * dzeta * (1 - fm), o1 = kz * dzeta * (1 + fm);
    l_kz += (lo[0] * o0 + lo[1] * o1) / kz;
    l_dzeta += lo[0] * 8 * kz * (1 - fm) + lo[1] * kz * (1 + fm);
    l_fm += -lo[0] * 8 * kz * dzeta + lo[1] * kz * dzeta;
    const T S2 = T(0.5) * drho * beta - T(0.25) * dzeta * drho;
    const T S3 = T(0.5) * drho * co + T(0.25) * dzeta * drho;
    l_kr += 2 * (lo[2] * S2 + lo[3] * S3);
    const T lS2 = 2 * kr * lo[2], lS3 = 2 * kr * lo[3];
    l_drho += lS2 * (T(0.5) * beta - T(0.25) * dzeta) + lS3 * (T(0.5) * co + T(0.25) * dzeta);
    l_dzeta += -lS2 * T(0.25) * drho + lS3 * T(0.25) * drho;
    l_beta += lS2 * T(0.5) * drho;
    l_co_direct += lS3 * T(0.5) * drho;
  }
  // drho = an - ao, dzeta = cn - co, fm = (ao + an)/2, beta = 1 - co
  l_an += l_drho + T(0.5) * l_fm;
  l_ao += -l_drho + T(0.5) * l_fm;
  l_cn += l_dzeta;
  l_co += -l_dzeta - l_beta + l_co_direct;
}

// ------------------------------------------------------------------ gather

template <typename T>
PDP3_HD void gather_weights(Tape<T> &tp) {
  const int i = tp.i, k = tp.k;
  const T a = tp.a, b = tp.b;
  int ir = a > T(0.5) ? i : i - 1;
  if (ir < 0) ir = 0;
  tp.ir_h = ir;
  {
    const T d21 = T(ir - i) + T(1.5) - a, s21 = T(ir + i) + T(0.5) + a;
    const T d32 = T(i - ir) + a - T(0.5), s32 = T(i + ir) + T(1.5) + a;
    tp.wrh[0] = d21 * s21 / (2 * T(ir + 1));
    tp.wrh[1] = d32 * s32 / (2 * T(ir + 3));
    tp.dwrh[0] = (d21 - s21) / (2 * T(ir + 1));
    tp.dwrh[1] = (s32 + d32) / (2 * T(ir + 3));
  }
  {
    const T fi = T(i), v1 = i >= 1 ? 2 * fi : T(0.25);
    tp.wrn[0] = (1 - a) * (2 * fi + a) / v1;
    tp.wrn[1] = a * (2 * fi + 1 + a) / (2 * (fi + 2));
    tp.dwrn[0] = (1 - 2 * fi - 2 * a) / v1;
    tp.dwrn[1] = (2 * fi + 1 + 2 * a) / (2 * (fi + 2));
  }
  int kz = b > T(0.5) ? k : k - 1;
  if (kz < 0) kz = 0;
  tp.kz_h = kz;
  tp.wzh[0] = T(kz - k) + T(1.5) - b;
  tp.wzh[1] = T(k - kz) + b - T(0.5);
  tp.wzn[0] = 1 - b;
  tp.wzn[1] = b;
}

// component c of E (0 r, 1 phi, 2 z) and H: which radial / axial weights
// (E_r: rhalf,znode; E_phi: rnode,znode; E_z: rnode,zhalf;
//  H_r: rnode,zhalf; H_phi: rhalf,zhalf; H_z: rhalf,znode)
PDP3_HD int comp_rhalf(int field, int c) {
  return field == 0 ? (c == 0) : (c != 0);
}
PDP3_HD int comp_zhalf(int field, int c) {
  return field == 0 ? (c == 2) : (c != 2);
}

template <typename T>
PDP3_HD T interp(const Tape<T> &tp, T f0, T f1, T f2, T f3, bool rh, bool zh) {
  // value selects (no pointer into the tape), so the tape can stay in registers
  const T wr0 = rh ? tp.wrh[0] : tp.wrn[0], wr1 = rh ? tp.wrh[1] : tp.wrn[1];
  const T wz0 = zh ? tp.wzh[0] : tp.wzn[0], wz1 = zh ? tp.wzh[1] : tp.wzn[1];
  return wz0 * (f0 * wr0 + f1 * wr1) + wz1 * (f2 * wr0 + f3 * wr1);
}

// ----------------------------------------------------------------- forward

template <typename T>
PDP3_HD void renorm_t(int &i, T &f) {
  for (int it = 0; it < 4 && f > T(1); it++) { f -= T(1); i += 1; }
  for (int it = 0; it < 4 && f <= T(0); it++) { f += T(1); i -= 1; }
  if (i < 0) { f = f + T(i); i = 0; }
}

// tp.{i,k,a,b,u,w,fe,fh} set by the caller; fills the rest.  Deposits are
// not applied here (the forward kernel already did); the adjoint needs
// their node positions only.
template <typename T>
PDP3_HD void forward(const Consts<T> &C, Tape<T> &tp) {
  gather_weights(tp);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    tp.e[c] = interp(tp, tp.fe[c][0], tp.fe[c][1], tp.fe[c][2], tp.fe[c][3], comp_rhalf(0, c),
                     comp_zhalf(0, c));
    tp.h[c] = interp(tp, tp.fh[c][0], tp.fh[c][1], tp.fh[c][2], tp.fh[c][3], comp_rhalf(1, c),
                     comp_zhalf(1, c));
  }
  // Boris, relativistic
#pragma unroll
  for (int c = 0; c < 3; c++) tp.um[c] = tp.u[c] + C.ke * tp.e[c];
  tp.gi = T(1) / sqrt(T(1) + tp.um[0] * tp.um[0] + tp.um[1] * tp.um[1] + tp.um[2] * tp.um[2]);
#pragma unroll
  for (int c = 0; c < 3; c++) tp.tb[c] = C.kb * tp.h[c] * tp.gi;
  tp.c2 = T(2) / (T(1) + tp.tb[0] * tp.tb[0] + tp.tb[1] * tp.tb[1] + tp.tb[2] * tp.tb[2]);
  tp.wv[0] = tp.um[0] + (tp.um[1] * tp.tb[2] - tp.um[2] * tp.tb[1]);
  tp.wv[1] = tp.um[1] + (tp.um[2] * tp.tb[0] - tp.um[0] * tp.tb[2]);
  tp.wv[2] = tp.um[2] + (tp.um[0] * tp.tb[1] - tp.um[1] * tp.tb[0]);
  tp.v2[0] = tp.wv[1] * tp.tb[2] - tp.wv[2] * tp.tb[1];
  tp.v2[1] = tp.wv[2] * tp.tb[0] - tp.wv[0] * tp.tb[2];
  tp.v2[2] = tp.wv[0] * tp.tb[1] - tp.wv[1] * tp.tb[0];
#pragma unroll
  for (int c = 0; c < 3; c++) tp.up[c] = tp.um[c] + tp.c2 * tp.v2[c] + C.ke * tp.e[c];
  tp.inv_g = T(1) / sqrt(T(1) + tp.up[0] * tp.up[0] + tp.up[1] * tp.up[1] + tp.up[2] * tp.up[2]);
#pragma unroll
  for (int c = 0; c < 3; c++) tp.vel[c] = tp.up[c] * tp.inv_g;
  // first half move, rz rotation
  tp.dr_h = tp.vel[0] * C.cr;
  tp.dy = tp.vel[1] * C.cr;
  tp.dz_h = tp.vel[2] * C.cz;
  tp.x = T(tp.i) + tp.a + tp.dr_h;
  tp.rr = sqrt(tp.x * tp.x + tp.dy * tp.dy);
  tp.b1 = tp.b + tp.dz_h;
  {
    int i1 = tp.i, k1 = tp.k;
    T f1 = tp.rr - T(tp.i), g1 = tp.b1;
    renorm_t(i1, f1);
    renorm_t(k1, g1);
    tp.i1 = i1;
    tp.k1 = k1;
    tp.f1 = f1;
    tp.g1 = g1;
    const T fi1 = T(i1), rho1 = fi1 + f1, v1 = i1 >= 1 ? 2 * fi1 : T(0.25);
    const T Na = (1 - f1) * (2 * fi1 + f1), Nb = f1 * (2 * fi1 + 1 + f1);
    const T Db = rho1 * 2 * (fi1 + 1);
    tp.wa = Na / (rho1 * v1);
    tp.wb = Nb / Db;
    tp.dwa = ((1 - 2 * fi1 - 2 * f1) * rho1 - Na) / (rho1 * rho1 * v1);
    tp.dwb = ((2 * fi1 + 1 + 2 * f1) * rho1 - Nb) / (rho1 * Db);
    tp.pref = C.kphi * tp.w * tp.vel[1];
  }
  // second half move and walls (positions relative to the start cell)
  T xa2 = tp.rr - T(tp.i) + tp.dr_h, b2 = tp.b1 + tp.dz_h;
  tp.sr = 1;
  tp.sz = 1;
  tp.ur_sign = 1;
  tp.uz_sign = 1;
  tp.alive_now = true;
  const T wr_rel = T(C.nr - 1) - T(0.5) - T(tp.i), wz_rel = T(C.nz - 1) - T(0.5) - T(tp.k);
  if (!C.bunch) {
    if (xa2 > wr_rel) { xa2 = 2 * wr_rel - xa2; tp.sr = -tp.sr; tp.ur_sign = -tp.ur_sign; }
    if (b2 > wz_rel) { b2 = 2 * wz_rel - b2; tp.sz = -tp.sz; tp.uz_sign = -tp.uz_sign; }
  } else {
    if (xa2 > wr_rel) tp.alive_now = false;
    if (b2 > wz_rel) tp.alive_now = false;
  }
  if (xa2 < T(0.5) - T(tp.i)) { xa2 = 1 - 2 * T(tp.i) - xa2; tp.sr = -tp.sr; tp.ur_sign = -tp.ur_sign; }
  if (b2 < T(0.5) - T(tp.k)) { b2 = 1 - 2 * T(tp.k) - b2; tp.sz = -tp.sz; tp.uz_sign = -tp.uz_sign; }
  tp.x2 = T(tp.i) + xa2;
  tp.r2 = sqrt(tp.x2 * tp.x2 + tp.dy * tp.dy);
  tp.A = tp.r2 - T(tp.i);
  tp.B = b2;
  T an = tp.A, bn = tp.B;
  int in = tp.i, kn = tp.k;
  renorm_t(in, an);
  renorm_t(kn, bn);
  tp.in = in;
  tp.kn = kn;
  tp.an = an;
  tp.bn = bn;
  tp.st = tp.dy / tp.r2;
  tp.ct = tp.x2 / tp.r2;
  const T urf = tp.ur_sign * tp.up[0], uzf = tp.uz_sign * tp.up[2];
  if (tp.alive_now) {
    tp.uout[0] = tp.ct * urf - tp.st * tp.up[1];
    tp.uout[1] = tp.st * urf + tp.ct * tp.up[1];
  } else {
    tp.uout[0] = urf;
    tp.uout[1] = tp.up[1];
  }
  tp.uout[2] = uzf;
  // r-z path (particles_f32.cuh deposit_path)
  tp.path_ok = false;
  tp.np = 0;
  if (!tp.alive_now) return;
  const int di = in - tp.i, dk = kn - tp.k;
  if (di < -1 || di > 1 || dk < -1 || dk > 1) return;
  tp.path_ok = true;
  if (di == 0 && dk == 0) {
    // the step stays in its cell: one piece from (a, b) to (an, bn)
    tp.qa0 = tp.a;
    tp.qb0 = tp.b;
    tp.qa1 = an;
    tp.qb1 = bn;
    tp.pci0 = tp.i;
    tp.pck0 = tp.k;
    return;
  }
  const T A = T(di) + an, B = T(dk) + bn;
  T tr = 2, tz = 2;
  if (di != 0) tr = ((di > 0 ? T(1) : T(0)) - tp.a) / (A - tp.a);
  if (dk != 0) tz = ((dk > 0 ? T(1) : T(0)) - tp.b) / (B - tp.b);
  tp.ts0 = tp.ts1 = T(2);
  tp.kind0 = tp.kind1 = 0;
  if (tr <= T(1) && tz <= T(1)) {
    if (tr <= tz) { tp.ts0 = tr; tp.kind0 = 0; tp.ts1 = tz; tp.kind1 = 1; }
    else { tp.ts0 = tz; tp.kind0 = 1; tp.ts1 = tr; tp.kind1 = 0; }
    tp.np = 2;
  } else if (tr <= T(1)) {
    tp.ts0 = tr; tp.kind0 = 0; tp.np = 1;
  } else if (tz <= T(1)) {
    tp.ts0 = tz; tp.kind0 = 1; tp.np = 1;
  }
  // crossing point p: the crossed coordinate sits on the face
  const T fa = di > 0 ? T(1) : T(0), fb = dk > 0 ? T(1) : T(0);
  const T ca0 = tp.kind0 == 0 ? fa : tp.a + tp.ts0 * (A - tp.a);
  const T cb0 = tp.kind0 == 0 ? tp.b + tp.ts0 * (B - tp.b) : fb;
  const T ca1 = tp.kind1 == 0 ? fa : tp.a + tp.ts1 * (A - tp.a);
  const T cb1 = tp.kind1 == 0 ? tp.b + tp.ts1 * (B - tp.b) : fb;
  tp.qa0 = tp.a;
  tp.qb0 = tp.b;
  tp.qa1 = tp.np >= 1 ? ca0 : A;
  tp.qb1 = tp.np >= 1 ? cb0 : B;
  tp.qa2 = tp.np >= 2 ? ca1 : A;
  tp.qb2 = tp.np >= 2 ? cb1 : B;
  tp.qa3 = A;
  tp.qb3 = B;
  tp.pci0 = tp.i;
  tp.pck0 = tp.k;
  tp.pci1 = tp.pci0 + (tp.np >= 1 && tp.kind0 == 0 ? di : 0);
  tp.pck1 = tp.pck0 + (tp.np >= 1 && tp.kind0 == 1 ? dk : 0);
  tp.pci2 = tp.pci1 + (tp.np >= 2 && tp.kind1 == 0 ? di : 0);
  tp.pck2 = tp.pck1 + (tp.np >= 2 && tp.kind1 == 1 ? dk : 0);
}

// Deposit values of the particle's pieces (for checks): jz/jr per piece
template <typename T>
PDP3_HD void piece_outputs(const Consts<T> &C, const Tape<T> &tp, int p, T out[4]) {
  const T oi = T(tp.pci(p) - tp.i), ok = T(tp.pck(p) - tp.k);
  piece_fwd(tp.pci(p), tp.qa(p) - oi, tp.qb(p) - ok, tp.qa(p + 1) - oi, tp.qb(p + 1) - ok,
            C.kz * tp.w, C.kr * tp.w, out);
}

// ------------------------------------------------------- gather jump terms

// The radial gather weights are discontinuous in r (the upstream normalises
// the outer node of a node-centred component by CELL_VOLUME(i+2) and switches
// the inner node of a half-node component at the cell middle), so the mean
// field that many particles see moves with a shift of the particles by the
// jumps times the particle density at the jumps, a term no single particle's
// derivative contains.  With the density taken uniform inside a cell, each
// particle carries the expected share per unit offset:
//   node-centred (E_phi, E_z, H_r): half the jump at each face of its cell,
//     jump at the face between cells i and i+1 = f_{i+1} / (i + 2);
//   half-node (E_r, H_phi, H_z), i >= 1: the jump at the cell middle,
//     f_i (2i + 1) / (2 (i + 1)(i + 2)).
// f_j is the node row's value interpolated in z with the particle's weights.
// wall_cells: the walls reflect whatever ends a step at r < dr/2 or
// r > r_max - dr/2, so the axis cell and the last cell hold their particles
// in the half next to the other cells, twice as dense: there a particle
// carries the whole jump of the face on that side and none of the other.
// face_h > 0 replaces the uniform-density shares by a box-kernel estimate
// of the density at each jump: a particle within face_h (in cells) of a jump
// carries that jump / (2 face_h), others none of it.  In expectation this
// equals the uniform shares where the density is linear inside the cell,
// and it follows the density where it is not (a wake's compressed electrons,
// half-filled wall cells).
template <typename T>
PDP3_HD T radial_jump(const Tape<T> &tp, T f0, T f1, T f2, T f3, T wz0, T wz1, bool rh,
                      bool wall_cells, int nr, T face_h) {
  const int i = tp.i;
  const T lo = wz0 * f0 + wz1 * f2, hi = wz0 * f1 + wz1 * f3;
  if (!rh) {
    // nodes i, i+1: top face jump uses f_{i+1}, bottom face (i >= 1) f_i
    const T top = hi / T(i + 2);
    const T bottom = i >= 1 ? lo / T(i + 1) : T(0);
    if (face_h > T(0)) {
      T s = T(0);
      if (tp.a > T(1) - face_h) s += top / (T(2) * face_h);
      if (tp.a < face_h) s += bottom / (T(2) * face_h);
      return s;
    }
    if (wall_cells && i == 0) return top;
    if (wall_cells && i == nr - 2) return bottom;
    return T(0.5) * (top + bottom);
  }
  if (i < 1) return T(0);
  const T fi = tp.ir_h == i ? lo : hi;  // node i is the inner node when ir = i
  const T jump = fi * T(2 * i + 1) / (T(2) * T(i + 1) * T(i + 2));
  if (face_h > T(0)) {
    const T d = tp.a - T(0.5);  // the jump sits at the cell middle
    return (d < face_h && d > -face_h) ? jump / (T(2) * face_h) : T(0);
  }
  return jump;
}

// adjoint of one gathered component: lv = adjoint of the gathered value;
// writes the adjoints of its four node values and adds the position terms
template <typename T>
PDP3_HD void gather_rev(const Consts<T> &C, const Tape<T> &tp, const T f[4], bool rh, bool zh,
                        T lv, T lf[4], T &l_a, T &l_b) {
  const T wr0 = rh ? tp.wrh[0] : tp.wrn[0], wr1 = rh ? tp.wrh[1] : tp.wrn[1];
  const T dwr0 = rh ? tp.dwrh[0] : tp.dwrn[0], dwr1 = rh ? tp.dwrh[1] : tp.dwrn[1];
  const T wz0 = zh ? tp.wzh[0] : tp.wzn[0], wz1 = zh ? tp.wzh[1] : tp.wzn[1];
  const T f0 = f[0], f1 = f[1], f2 = f[2], f3 = f[3];
  lf[0] = lv * wz0 * wr0;
  lf[1] = lv * wz0 * wr1;
  lf[2] = lv * wz1 * wr0;
  lf[3] = lv * wz1 * wr1;
  l_a += lv * (wz0 * (f0 * dwr0 + f1 * dwr1) + wz1 * (f2 * dwr0 + f3 * dwr1));
  // d wz0 / db = -1, d wz1 / db = +1 for both the node and the half-node weights
  l_b += lv * (-(f0 * wr0 + f1 * wr1) + (f2 * wr0 + f3 * wr1));
  if (C.face & 1)
    l_a += lv * radial_jump(tp, f0, f1, f2, f3, wz0, wz1, rh, C.face & 4, C.nr, C.face_h);
}

// The walls reflect a particle whose end point lies beyond them: the end
// point is mirrored (continuous where it meets the wall) and u_r or u_z
// changes sign, a jump of the output momentum at the start offset a* (b*)
// whose end point lies on the wall.  The deposits are continuous there.  A
// particle carries per unit offset S(a*+) - S(a*-) for each such a* inside
// its cell, times the expected density there, S the adjoint-weighted output
// momentum with the end point on the wall:
//   radial: rr = sqrt(x^2 + dy^2), x = i + a + dr_h; the axis reflects where
//     rr < 1/2 - dr_h (thresholds x = +-s), the outer wall where
//     rr > nr - 3/2 - dr_h; S(refl) - S(unrefl) = -2 u_r (ct l_ur' + st l_uphi')
//     with (ct, st) the rotation of the end point on the wall;
//   z: b2 = b + 2 dz_h; S(refl) - S(unrefl) = -2 u_z l_uz'.
// Density: uniform inside a cell, except that no particle stays beyond a
// wall (r < dr/2, z < dz/2, r > r_max - dr/2, z > z_max - dz/2: the first step
// reflects it, and injected bunch particles start at z >= dz/2), so a wall
// cell holds its particles in its inner half at twice the density, and a
// threshold in its outer half carries nothing.  Bunch particles that leave
// through the outer walls are removed, which has no linear jump; those walls
// count for plasma species only.
template <typename T>
PDP3_HD T wall_density(T t, bool low_wall, bool high_wall) {
  if (!(t > T(0) && t < T(1))) return T(0);
  if (low_wall) return t > T(0.5) ? T(2) : T(0);
  if (high_wall) return t < T(0.5) ? T(2) : T(0);
  return T(1);
}

template <typename T>
PDP3_HD T radial_wall_dS(const Tape<T> &tp, const T l_uout[3], T x2w) {
  const T r2w = sqrt(x2w * x2w + tp.dy * tp.dy);
  return T(-2) * tp.up[0] * (x2w / r2w * l_uout[0] + tp.dy / r2w * l_uout[1]);
}

template <typename T>
PDP3_HD void wall_jumps(const Consts<T> &C, const Tape<T> &tp, const T l_uout[3], T &l_a,
                        T &l_b) {
  const bool axis_cell = tp.i == 0, outer_cell = tp.i == C.nr - 2;
  const bool left_cell = tp.k == 0, right_cell = tp.k == C.nz - 2;
  const T off = T(tp.i) + tp.dr_h, dy2 = tp.dy * tp.dy;
  const T Ra = T(0.5) - tp.dr_h;
  if (Ra * Ra > dy2) {
    const T s = sqrt(Ra * Ra - dy2), dS = radial_wall_dS(tp, l_uout, T(0.5));
    // rr rises with a at x = s (reflected below a*), falls at x = -s
    l_a -= dS * wall_density(s - off, axis_cell, outer_cell);
    l_a += dS * wall_density(-s - off, axis_cell, outer_cell);
  }
  const T Ro = T(C.nr) - T(1.5) - tp.dr_h;
  if (!C.bunch && Ro * Ro > dy2) {
    const T ao = sqrt(Ro * Ro - dy2) - off;
    l_a += radial_wall_dS(tp, l_uout, T(C.nr) - T(1.5)) * wall_density(ao, axis_cell, outer_cell);
  }
  const T dSz = T(-2) * tp.up[2] * l_uout[2];
  l_b -= dSz * wall_density(T(0.5) - T(tp.k) - 2 * tp.dz_h, left_cell, right_cell);
  if (!C.bunch)
    l_b += dSz * wall_density(T(C.nz) - T(1.5) - T(tp.k) - 2 * tp.dz_h, left_cell, right_cell);
}

// ----------------------------------------------------------------- reverse

// Inputs: l_an, l_bn, l_uout[3] (adjoints of the stored outputs), l_jphi[4]
// (adjoint of J_phi at (i1,k1),(i1+1,k1),(i1,k1+1),(i1+1,k1+1)), l_piece[p][4]
// (adjoint of J_z(ci,ck), J_z(ci+1,ck), J_r(ci,ck), J_r(ci,ck+1) per piece).
// Outputs: l_a, l_b, l_u[3], l_w, l_fe[3][4], l_fh[3][4].
// WALLS = false compiles the wall terms out (C.face bit 1 is then ignored),
// which keeps them from costing registers where they are off.
template <typename T, bool WALLS = true>
PDP3_HD void reverse(const Consts<T> &C, const Tape<T> &tp, T l_an, T l_bn, const T l_uout[3],
                     const T l_jphi[4], const T l_piece[3][4], T &l_a, T &l_b, T l_u[3], T &l_w,
                     T l_fe[3][4], T l_fh[3][4]) {
  T l_up[3] = {0, 0, 0}, l_e[3] = {0, 0, 0}, l_h[3] = {0, 0, 0};
  T l_rr = 0, l_dy = 0, l_b1 = 0, l_dr = 0, l_dz = 0, l_vel[3] = {0, 0, 0};
  l_a = 0;
  l_b = 0;
  l_w = 0;
  if (WALLS && (C.face & 2)) wall_jumps(C, tp, l_uout, l_a, l_b);
  // ---- outputs: an = A - shift, bn = B - shift; rotation of u
  T l_A = tp.alive_now ? l_an : T(0), l_B = tp.alive_now ? l_bn : T(0);
  T l_x2 = 0, l_r2 = 0;
  const T urf = tp.ur_sign * tp.up[0];
  if (tp.alive_now) {
    const T l_ct = l_uout[0] * urf + l_uout[1] * tp.up[1];
    const T l_st = -l_uout[0] * tp.up[1] + l_uout[1] * urf;
    const T l_urf = tp.ct * l_uout[0] + tp.st * l_uout[1];
    l_up[1] += -tp.st * l_uout[0] + tp.ct * l_uout[1];
    l_up[0] += tp.ur_sign * l_urf;
    l_up[2] += tp.uz_sign * l_uout[2];
    l_x2 += l_ct / tp.r2;
    l_r2 += -l_ct * tp.ct / tp.r2 - l_st * tp.st / tp.r2;
    l_dy += l_st / tp.r2;
    // ---- r-z path adjoint
    if (tp.path_ok && tp.np == 0) {
      // the step stays in its cell (almost every step): one piece from
      // (a, b) to (A, B), the general loop's single iteration
      const T lo[4] = {l_piece[0][0], l_piece[0][1], l_piece[0][2], l_piece[0][3]};
      T la0 = 0, lc0 = 0, la1 = 0, lc1 = 0, lkz = 0, lkr = 0;
      piece_rev(tp.i, tp.qa0, tp.qb0, tp.qa1, tp.qb1, C.kz * tp.w, C.kr * tp.w, lo, la0, lc0,
                la1, lc1, lkz, lkr);
      l_w += lkz * C.kz + lkr * C.kr;
      l_a += la0;
      l_b += lc0;
      l_A += la1;
      l_B += lc1;
    } else if (tp.path_ok) {
      // adjoints of the path points Q0..Q3, kept in scalars: the piece loop is
      // not unrolled (one copy of piece_rev) and reads the tape through
      // selects, so nothing is indexed at run time
      T lqa0 = 0, lqa1 = 0, lqa2 = 0, lqa3 = 0, lqb0 = 0, lqb1 = 0, lqb2 = 0, lqb3 = 0;
#pragma unroll 1
      for (int p = 0; p <= tp.np; p++) {
        const int pci = tp.pci(p), pck = tp.pck(p);
        const T oi = T(pci - tp.i), ok = T(pck - tp.k);
        const T qa0 = tp.qa(p), qb0 = tp.qb(p), qa1 = tp.qa(p + 1), qb1 = tp.qb(p + 1);
        const T lo[4] = {sel3(p, l_piece[0][0], l_piece[1][0], l_piece[2][0]),
                         sel3(p, l_piece[0][1], l_piece[1][1], l_piece[2][1]),
                         sel3(p, l_piece[0][2], l_piece[1][2], l_piece[2][2]),
                         sel3(p, l_piece[0][3], l_piece[1][3], l_piece[2][3])};
        T la0 = 0, lc0 = 0, la1 = 0, lc1 = 0, lkz = 0, lkr = 0;
        piece_rev(pci, qa0 - oi, qb0 - ok, qa1 - oi, qb1 - ok, C.kz * tp.w, C.kr * tp.w, lo,
                  la0, lc0, la1, lc1, lkz, lkr);
        // Q_p gets (la0, lc0), Q_{p+1} gets (la1, lc1)
        lqa0 += p == 0 ? la0 : T(0);
        lqa1 += p == 1 ? la0 : (p == 0 ? la1 : T(0));
        lqa2 += p == 2 ? la0 : (p == 1 ? la1 : T(0));
        lqa3 += p == 2 ? la1 : T(0);
        lqb0 += p == 0 ? lc0 : T(0);
        lqb1 += p == 1 ? lc0 : (p == 0 ? lc1 : T(0));
        lqb2 += p == 2 ? lc0 : (p == 1 ? lc1 : T(0));
        lqb3 += p == 2 ? lc1 : T(0);
        l_w += lkz * C.kz + lkr * C.kr;
      }
      // crossing points depend on P0 = (a, b) and P1 = (A, B)
      const int di = tp.in - tp.i, dk = tp.kn - tp.k;
      const T Ar = T(di) + tp.an, Br = T(dk) + tp.bn;  // = A, B relative to the start cell
#pragma unroll 1
      for (int p = 1; p <= tp.np; p++) {
        const T t = tp.ts(p - 1);
        if (tp.kind(p - 1) == 0) {
          // qb = b + t (B - b), t = (fr - a)/(A - a)
          const T fr = di > 0 ? T(1) : T(0), den = Ar - tp.a;
          const T dt_da = (-(den) + (fr - tp.a)) / (den * den), dt_dA = -(fr - tp.a) / (den * den);
          const T l = p == 1 ? lqb1 : lqb2;
          l_b += l * (1 - t);
          l_B += l * t;
          l_a += l * (Br - tp.b) * dt_da;
          l_A += l * (Br - tp.b) * dt_dA;
        } else {
          const T fz = dk > 0 ? T(1) : T(0), den = Br - tp.b;
          const T dt_db = (-(den) + (fz - tp.b)) / (den * den), dt_dB = -(fz - tp.b) / (den * den);
          const T l = p == 1 ? lqa1 : lqa2;
          l_a += l * (1 - t);
          l_A += l * t;
          l_b += l * (Ar - tp.a) * dt_db;
          l_B += l * (Ar - tp.a) * dt_dB;
        }
      }
      l_a += lqa0;
      l_b += lqb0;
      l_A += tp.np == 0 ? lqa1 : (tp.np == 1 ? lqa2 : lqa3);
      l_B += tp.np == 0 ? lqb1 : (tp.np == 1 ? lqb2 : lqb3);
    }
  } else {
    l_up[0] += tp.ur_sign * l_uout[0];
    l_up[1] += l_uout[1];
    l_up[2] += tp.uz_sign * l_uout[2];
  }
  // A = r2 - i, B = b2 (after walls), r2 = sqrt(x2^2 + dy^2), x2 = i + xa2
  l_r2 += l_A;
  l_x2 += l_r2 * tp.x2 / tp.r2;
  l_dy += l_r2 * tp.dy / tp.r2;
  // xa2 = c + sr (rr - i + dr_h), b2 = c' + sz (b1 + dz_h)
  l_rr += tp.sr * l_x2;
  l_dr += tp.sr * l_x2;
  l_b1 += tp.sz * l_B;
  l_dz += tp.sz * l_B;
  // ---- j_phi: J = pref (1-g1) wa, pref (1-g1) wb, pref g1 wa, pref g1 wb
  {
    const T g1 = tp.g1;
    const T l_pref = l_jphi[0] * (1 - g1) * tp.wa + l_jphi[1] * (1 - g1) * tp.wb +
                     l_jphi[2] * g1 * tp.wa + l_jphi[3] * g1 * tp.wb;
    const T l_g1 = tp.pref * (-l_jphi[0] * tp.wa - l_jphi[1] * tp.wb + l_jphi[2] * tp.wa +
                              l_jphi[3] * tp.wb);
    const T l_wa = tp.pref * ((1 - g1) * l_jphi[0] + g1 * l_jphi[2]);
    const T l_wb = tp.pref * ((1 - g1) * l_jphi[1] + g1 * l_jphi[3]);
    l_rr += l_wa * tp.dwa + l_wb * tp.dwb;  // f1 = rr - i1
    l_b1 += l_g1;                          // g1 = b1 - shift
    l_w += l_pref * C.kphi * tp.vel[1];
    l_vel[1] += l_pref * C.kphi * tp.w;
  }
  // ---- first half move: rr = sqrt(x^2 + dy^2), x = i + a + dr_h, b1 = b + dz_h
  {
    const T l_x = l_rr * tp.x / tp.rr;
    l_dy += l_rr * tp.dy / tp.rr;
    l_a += l_x;
    l_dr += l_x;
    l_b += l_b1;
    l_dz += l_b1;
  }
  // dr_h = vel_r cr, dy = vel_phi cr, dz_h = vel_z cz
  l_vel[0] += l_dr * C.cr;
  l_vel[1] += l_dy * C.cr;
  l_vel[2] += l_dz * C.cz;
  // vel = up inv_g, inv_g = (1 + |up|^2)^(-1/2)
  {
    T l_ig = 0;
    for (int c = 0; c < 3; c++) {
      l_up[c] += l_vel[c] * tp.inv_g;
      l_ig += l_vel[c] * tp.up[c];
    }
    const T g3 = tp.inv_g * tp.inv_g * tp.inv_g;
    for (int c = 0; c < 3; c++) l_up[c] += -l_ig * g3 * tp.up[c];
  }
  // ---- Boris reverse: up = um + c2 v2 + ke e
  T l_um[3], l_v2[3], l_wv[3] = {0, 0, 0}, l_tb[3] = {0, 0, 0}, l_c2 = 0, l_gi = 0;
  for (int c = 0; c < 3; c++) {
    l_um[c] = l_up[c];
    l_v2[c] = tp.c2 * l_up[c];
    l_c2 += l_up[c] * tp.v2[c];
    l_e[c] += C.ke * l_up[c];
  }
  // v2 = wv x tb: l_wv += tb x l_v2, l_tb += l_v2 x wv
  l_wv[0] += tp.tb[1] * l_v2[2] - tp.tb[2] * l_v2[1];
  l_wv[1] += tp.tb[2] * l_v2[0] - tp.tb[0] * l_v2[2];
  l_wv[2] += tp.tb[0] * l_v2[1] - tp.tb[1] * l_v2[0];
  l_tb[0] += l_v2[1] * tp.wv[2] - l_v2[2] * tp.wv[1];
  l_tb[1] += l_v2[2] * tp.wv[0] - l_v2[0] * tp.wv[2];
  l_tb[2] += l_v2[0] * tp.wv[1] - l_v2[1] * tp.wv[0];
  // wv = um + um x tb: l_um += l_wv + tb x l_wv, l_tb += l_wv x um
  for (int c = 0; c < 3; c++) l_um[c] += l_wv[c];
  l_um[0] += tp.tb[1] * l_wv[2] - tp.tb[2] * l_wv[1];
  l_um[1] += tp.tb[2] * l_wv[0] - tp.tb[0] * l_wv[2];
  l_um[2] += tp.tb[0] * l_wv[1] - tp.tb[1] * l_wv[0];
  l_tb[0] += l_wv[1] * tp.um[2] - l_wv[2] * tp.um[1];
  l_tb[1] += l_wv[2] * tp.um[0] - l_wv[0] * tp.um[2];
  l_tb[2] += l_wv[0] * tp.um[1] - l_wv[1] * tp.um[0];
  // c2 = 2 / (1 + |tb|^2): l_tb += l_c2 (-c2^2) tb
  for (int c = 0; c < 3; c++) l_tb[c] += -l_c2 * tp.c2 * tp.c2 * tp.tb[c];
  // tb = kb h gi
  for (int c = 0; c < 3; c++) {
    l_h[c] += l_tb[c] * C.kb * tp.gi;
    l_gi += l_tb[c] * C.kb * tp.h[c];
  }
  // gi = (1 + |um|^2)^(-1/2)
  {
    const T g3 = tp.gi * tp.gi * tp.gi;
    for (int c = 0; c < 3; c++) l_um[c] += -l_gi * g3 * tp.um[c];
  }
  // um = u + ke e
  for (int c = 0; c < 3; c++) {
    l_u[c] = l_um[c];
    l_e[c] += C.ke * l_um[c];
  }
  // ---- gather reverse: field-node adjoints and position dependence
#pragma unroll
  for (int c = 0; c < 3; c++) {
    gather_rev(C, tp, tp.fe[c], comp_rhalf(0, c), comp_zhalf(0, c), l_e[c], l_fe[c], l_a, l_b);
    gather_rev(C, tp, tp.fh[c], comp_rhalf(1, c), comp_zhalf(1, c), l_h[c], l_fh[c], l_a, l_b);
  }
}

}  // namespace adj
}  // namespace pdp3g
