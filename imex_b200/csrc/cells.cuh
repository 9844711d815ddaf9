// Per-cell bodies of the stencil sub-steps, templated on the scalar type S and on a
// loader ld(a, k, m) that returns plane k of input array a at cell m.  The forward
// kernels instantiate them with S = double and plain loads (the operations and their
// order are the reference's); the adjoint instantiates them with Dual<L> and a loader
// that seeds L of the inputs, which yields L columns of the cell's Jacobian.
#pragma once

#include "device_common.cuh"

namespace imex {

// the 3x3 neighbourhood of cell (i, j) (periodic images or clamped cells, cid): nb[(dj + 1) * 3 + (di + 1)]
enum { NB_SW = 0, NB_S, NB_SE, NB_W, NB_C, NB_E, NB_NW, NB_N, NB_NE };
__device__ __forceinline__ void neighbours(const DevParams& P, int i, int j, long long* nb) {
#pragma unroll
  for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
    for (int di = -1; di <= 1; ++di) nb[(dj + 1) * 3 + (di + 1)] = cid(P, i + di, j + dj);
}
__device__ __forceinline__ void neighbours(const DevParams& P, long long n, long long* nb) {
  int i, j;
  cell_of(P, n, i, j);
  neighbours(P, i, j, nb);
}

// ---- B* right-hand side of MagSubsystem_UpdateB (imex_subsystems.cpp:549-615)
enum { MR_UCON = 0, MR_QE = 1, MR_PE = 2, MR_QS = 3 };
template <class S, class Ld>
__device__ __forceinline__ void mag_rhs_B_cell(const DevParams& P, double h, const long long* nb, Ld& ld, S* out) {
  const long long n = nb[NB_C], E = nb[NB_E], W = nb[NB_W], No = nb[NB_N], S_ = nb[NB_S];
  const long long NE = nb[NB_NE], SE = nb[NB_SE], NW = nb[NB_NW], SW = nb[NB_SW];
  const double dx = P.dx, dy = P.dy;
  auto U = [&](int k, long long m) { return ld(MR_UCON, k, m); };
  auto Q = [&](int k, long long m) { return ld(MR_QE, k, m); };
  auto PE = [&](long long m) { return ld(MR_PE, 0, m); };
  const S rho_p0 = 0.5 * (U(0, n) + U(0, E)), rho_m0 = 0.5 * (U(0, n) + U(0, W));
  const S rho_0p = 0.5 * (U(0, n) + U(0, No)), rho_0m = 0.5 * (U(0, n) + U(0, S_));
  const S rvx_p0 = 0.5 * (U(1, n) + U(1, E)), rvx_m0 = 0.5 * (U(1, n) + U(1, W));
  const S rvx_0p = 0.5 * (U(1, n) + U(1, No)), rvx_0m = 0.5 * (U(1, n) + U(1, S_));
  const S rvy_p0 = 0.5 * (U(2, n) + U(2, E)), rvy_m0 = 0.5 * (U(2, n) + U(2, W));
  const S rvy_0p = 0.5 * (U(2, n) + U(2, No)), rvy_0m = 0.5 * (U(2, n) + U(2, S_));
  const S rvz_p0 = 0.5 * (U(3, n) + U(3, E)), rvz_m0 = 0.5 * (U(3, n) + U(3, W));
  const S rvz_0p = 0.5 * (U(3, n) + U(3, No)), rvz_0m = 0.5 * (U(3, n) + U(3, S_));
  const S p_pp = 0.25 * (PE(n) + PE(E) + PE(No) + PE(NE));
  const S p_pm = 0.25 * (PE(n) + PE(E) + PE(S_) + PE(SE));
  const S p_mp = 0.25 * (PE(n) + PE(W) + PE(No) + PE(NW));
  const S p_mm = 0.25 * (PE(n) + PE(W) + PE(S_) + PE(SW));
  const S Bxn_p0 = 0.5 * (Q(5, n) + Q(5, E)), Bxn_m0 = 0.5 * (Q(5, n) + Q(5, W));
  const S Bxn_0p = 0.5 * (Q(5, n) + Q(5, No)), Bxn_0m = 0.5 * (Q(5, n) + Q(5, S_));
  const S Byn_p0 = 0.5 * (Q(6, n) + Q(6, E)), Byn_m0 = 0.5 * (Q(6, n) + Q(6, W));
  const S Byn_0p = 0.5 * (Q(6, n) + Q(6, No)), Byn_0m = 0.5 * (Q(6, n) + Q(6, S_));
  const S Bzn_p0 = 0.5 * (Q(7, n) + Q(7, E)), Bzn_m0 = 0.5 * (Q(7, n) + Q(7, W));
  const S Bzn_0p = 0.5 * (Q(7, n) + Q(7, No)), Bzn_0m = 0.5 * (Q(7, n) + Q(7, S_));
  out[0] = ld(MR_QS, 5, n) - (h / dy) * ((Bxn_0p / rho_0p * (rvy_0p - (h / dy) * (PE(No) - PE(n))) -
                                          Byn_0p / rho_0p * (rvx_0p - h / dx * (p_pp - p_mp))) -
                                         (Bxn_0m / rho_0m * (rvy_0m - (h / dy) * (PE(n) - PE(S_))) -
                                          Byn_0m / rho_0m * (rvx_0m - h / dx * (p_pm - p_mm))));
  out[1] = ld(MR_QS, 6, n) - (h / dx) * ((Byn_p0 / rho_p0 * (rvx_p0 - (h / dx) * (PE(E) - PE(n))) -
                                          Bxn_p0 / rho_p0 * (rvy_p0 - h / dy * (p_pp - p_pm))) -
                                         (Byn_m0 / rho_m0 * (rvx_m0 - (h / dx) * (PE(n) - PE(W))) -
                                          Bxn_m0 / rho_m0 * (rvy_m0 - h / dy * (p_mp - p_mm))));
  const S Bz1 = ((Bzn_p0 / rho_p0 * (rvx_p0 - h / dx * (PE(E) - PE(n))) - Bxn_p0 / rho_p0 * (rvz_p0)) -
                 (Bzn_m0 / rho_m0 * (rvx_m0 - h / dx * (PE(n) - PE(W))) - Bxn_m0 / rho_m0 * (rvz_m0)));
  const S Bz2 = ((Bzn_0p / rho_0p * (rvy_0p - h / dy * (PE(No) - PE(n))) - Byn_0p / rho_0p * (rvz_0p)) -
                 (Bzn_0m / rho_0m * (rvy_0m - h / dy * (PE(n) - PE(S_))) - Byn_0m / rho_0m * (rvz_0m)));
  out[2] = ld(MR_QS, 7, n) - (h / dx) * Bz1 - (h / dy) * Bz2;
}

// ---- CollectMagFluxes (ct_flux.cpp:5-130), GLF: out = {Fx, Fy}; scalars bmax = {B_max_x, B_max_y}
enum { CF_UCON = 0, CF_QE = 1, CF_PE = 2 };
template <class S, class Ld>
__device__ __forceinline__ void collect_cell(const DevParams& P, double h, const S* bmax, const long long* nb, Ld& ld,
                                             S* out) {
  const long long n = nb[NB_C], E = nb[NB_E], W = nb[NB_W], No = nb[NB_N], S_ = nb[NB_S];
  const long long NE = nb[NB_NE], SE = nb[NB_SE], NW = nb[NB_NW];
  const double dx = P.dx, dy = P.dy;
  auto U = [&](int k, long long m) { return ld(CF_UCON, k, m); };
  auto Q = [&](int k, long long m) { return ld(CF_QE, k, m); };
  auto PE = [&](long long m) { return ld(CF_PE, 0, m); };
  const S rho_p0 = 0.5 * (U(0, n) + U(0, E)), rho_0p = 0.5 * (U(0, n) + U(0, No));
  const S rvx_p0 = 0.5 * (U(1, n) + U(1, E)), rvy_p0 = 0.5 * (U(2, n) + U(2, E));
  const S rvx_0p = 0.5 * (U(1, n) + U(1, No)), rvy_0p = 0.5 * (U(2, n) + U(2, No));
  const S p_pp = 0.25 * (PE(n) + PE(E) + PE(No) + PE(NE));
  const S p_pm = 0.25 * (PE(n) + PE(E) + PE(S_) + PE(SE));
  const S p_mp = 0.25 * (PE(n) + PE(W) + PE(No) + PE(NW));
  const S Bxn_p0 = 0.5 * (Q(5, n) + Q(5, E)), Byn_p0 = 0.5 * (Q(6, n) + Q(6, E));
  const S Bxn_0p = 0.5 * (Q(5, n) + Q(5, No)), Byn_0p = 0.5 * (Q(6, n) + Q(6, No));
#define C4(f, k, a, b2, c) (0.25 * (f(k, n) + f(k, a) + f(k, b2) + f(k, c)))
  const S Bxn_pp = C4(Q, 5, E, No, NE), Bxn_pm = C4(Q, 5, E, S_, SE), Bxn_mp = C4(Q, 5, W, No, NW);
  const S Byn_pp = C4(Q, 6, E, No, NE), Byn_pm = C4(Q, 6, E, S_, SE), Byn_mp = C4(Q, 6, W, No, NW);
  const S Bzn_pp = C4(Q, 7, E, No, NE), Bzn_pm = C4(Q, 7, E, S_, SE), Bzn_mp = C4(Q, 7, W, No, NW);
  const S Bx1_pp = C4(U, 5, E, No, NE), Bx1_pm = C4(U, 5, E, S_, SE), Bx1_mp = C4(U, 5, W, No, NW);
  const S By1_pp = C4(U, 6, E, No, NE), By1_pm = C4(U, 6, E, S_, SE), By1_mp = C4(U, 6, W, No, NW);
  const S Bz1_pp = C4(U, 7, E, No, NE), Bz1_pm = C4(U, 7, E, S_, SE), Bz1_mp = C4(U, 7, W, No, NW);
#undef C4
  auto QU = [&](long long m) { return 0.5 * (Q(5, m) * U(5, m) + Q(6, m) * U(6, m) + Q(7, m) * U(7, m)); };
  const S Fn_x = Byn_p0 / rho_p0 * (rvx_p0 - (h / dx) * (PE(E) - PE(n))) -
                 Bxn_p0 / rho_p0 * (rvy_p0 - (h / dy) * (p_pp - p_pm));
  const S By_1 = Byn_p0 / rho_p0 *
                 (-P.rdx * ((QU(E) - Q(5, E) * U(5, E)) - (QU(n) - Q(5, n) * U(5, n))) +
                  P.rdy * (Bxn_pp * By1_pp - Bxn_pm * By1_pm));
  const S By_2 = Bxn_p0 / rho_p0 *
                 (-P.rdx * (Q(5, E) * U(6, E) - Q(5, n) * U(6, n)) +
                  P.rdy * ((0.5 * (Bxn_pp * Bx1_pp + Byn_pp * By1_pp + Bzn_pp * Bz1_pp) - Byn_pp * By1_pp) -
                              (0.5 * (Bxn_pm * Bx1_pm + Byn_pm * By1_pm + Bzn_pm * Bz1_pm) - Byn_pm * By1_pm)));
  const S nu_x = bmax[0] * dx;
  const S Fdiff_x = -nu_x * (U(6, E) - U(6, n)) / dx;
  out[0] = Fn_x + h * (By_1 + By_2) + Fdiff_x;
  const S Fn_y = Bxn_0p / rho_0p * (rvy_0p - (h / dy) * (PE(No) - PE(n))) -
                 Byn_0p / rho_0p * (rvx_0p - (h / dx) * (p_pp - p_mp));
  const S Bx_1 = Bxn_0p / rho_0p *
                 (P.rdx * (Bxn_pp * By1_pp - Bxn_mp * By1_mp) -
                  P.rdy * ((QU(No) - Q(6, No) * U(6, No)) - (QU(n) - Q(6, n) * U(6, n))));
  const S Bx_2 = Byn_0p / rho_0p *
                 (P.rdx * ((0.5 * (Bxn_pp * Bx1_pp + Byn_pp * By1_pp + Bzn_pp * Bz1_pp) - Bxn_pp * Bx1_pp) -
                              (0.5 * (Bxn_mp * Bx1_mp + Byn_mp * By1_mp + Bzn_mp * Bz1_mp) - Bxn_mp * Bx1_mp)) -
                  P.rdy * (Q(6, No) * U(5, No) - Q(6, n) * U(5, n)));
  const S nu_y = bmax[1] * dy;
  const S Fdiff_y = -nu_y * (U(5, No) - U(5, n)) / dy;
  out[1] = Fn_y + h * (Bx_1 + Bx_2) + Fdiff_y;
}

// ---- pressure right-hand side b (imex_subsystems.cpp:123-169 first, 226-269 second); kin =
// momentum of the kinetic term, rv = rho v* of the enthalpy-flux divergence
enum { PR_UCON = 0, PR_HH = 1, PR_RV = 2, PR_KIN = 3 };
template <class S, class Ld>
__device__ __forceinline__ void pressure_rhs_cell(const DevParams& P, double h, const long long* nb, Ld& ld, S* out) {
  const long long n = nb[NB_C], e = nb[NB_E], w = nb[NB_W], no = nb[NB_N], s = nb[NB_S];
  const S u5 = ld(PR_UCON, 5, n), u6 = ld(PR_UCON, 6, n), u7 = ld(PR_UCON, 7, n);
  const S B2 = u5 * u5 + u6 * u6 + u7 * u7;
  const S h00 = ld(PR_HH, 0, n), hp0 = ld(PR_HH, 0, e), hm0 = ld(PR_HH, 0, w), h0p = ld(PR_HH, 0, no),
          h0m = ld(PR_HH, 0, s);
  const S p_star = ld(PR_UCON, 4, n) - 0.5 * B2;
  const S kx = ld(PR_KIN, 0, n), ky = ld(PR_KIN, 1, n), kz = ld(PR_KIN, 2, n);
  // every input before the first division, so that the loads are all in flight together
  const S rho = ld(PR_UCON, 0, n);
  const S rxe = ld(PR_RV, 0, e), rxn = ld(PR_RV, 0, n), rxw = ld(PR_RV, 0, w);
  const S ryo = ld(PR_RV, 1, no), ryn = ld(PR_RV, 1, n), rys = ld(PR_RV, 1, s);
  out[0] = p_star - 0.5 * (kx * kx + ky * ky + kz * kz) / rho -
           h * (P.rdx * (0.5 * (hp0 + h00) * 0.5 * (rxe + rxn) - 0.5 * (hm0 + h00) * 0.5 * (rxw + rxn)) +
                (P.rdy * (0.5 * (h0p + h00) * 0.5 * (ryo + ryn) - 0.5 * (h0m + h00) * 0.5 * (rys + ryn))));
}

// ---- momentum correction rho v = rho v* - h grad p (imex_subsystems.cpp:186-215)
enum { MO_P = 0, MO_RV = 1 };
template <class S, class Ld>
__device__ __forceinline__ void momentum_cell(const DevParams& P, double h, const long long* nb, Ld& ld, S* out) {
  const long long n = nb[NB_C];
  // every input before the divisions h / dx, h / dy
  const S pc = ld(MO_P, 0, n), pw = ld(MO_P, 0, nb[NB_W]), pe = ld(MO_P, 0, nb[NB_E]);
  const S ps = ld(MO_P, 0, nb[NB_S]), pn = ld(MO_P, 0, nb[NB_N]);
  const S r0 = ld(MO_RV, 0, n), r1 = ld(MO_RV, 1, n);
  const S flux_xm = 0.5 * (pw + pc), flux_xp = 0.5 * (pc + pe);
  out[0] = r0 - h / P.dx * (flux_xp - flux_xm);
  const S flux_ym = 0.5 * (ps + pc), flux_yp = 0.5 * (pc + pn);
  out[1] = r1 - h / P.dy * (flux_yp - flux_ym);
}

// ---- E = V(p) + KE + ME (DefinitionofU, imex_subsystems.cpp:286-302)
enum { ED_P = 0, ED_UCON = 1 };
template <class S, class Ld>
__device__ __forceinline__ void energy_define_cell(const DevParams& P, const long long* nb, Ld& ld, S* out) {
  const long long n = nb[NB_C];
  const S r = ld(ED_UCON, 0, n), m1 = ld(ED_UCON, 1, n), m2 = ld(ED_UCON, 2, n), m3 = ld(ED_UCON, 3, n);
  const S b5 = ld(ED_UCON, 5, n), b6 = ld(ED_UCON, 6, n), b7 = ld(ED_UCON, 7, n);
  out[0] = Vbase(P, ld(ED_P, 0, n), r) + 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / r + 0.5 * (b5 * b5 + b6 * b6 + b7 * b7);
}

// ---- E -= h div(h_e rho v) (ConservationofU, imex_subsystems.cpp:303-392): the energy is
// advanced by the central flux of the specific enthalpy h = e(rho, p) + p / rho carried by
// the corrected momentum, with p the pressure the solve returned (ghosts by index map)
enum { EC_P = 0, EC_UCON = 1 };
template <class S, class Ld>
__device__ __forceinline__ void energy_conservation_cell(const DevParams& P, double h, const long long* nb, Ld& ld,
                                                         S* out) {
  const long long n = nb[NB_C], E = nb[NB_E], W = nb[NB_W], No = nb[NB_N], S_ = nb[NB_S];
  const S p00 = ld(EC_P, 0, n), pp0 = ld(EC_P, 0, E), pm0 = ld(EC_P, 0, W), p0p = ld(EC_P, 0, No), p0m = ld(EC_P, 0, S_);
  const S r00 = ld(EC_UCON, 0, n), rp0 = ld(EC_UCON, 0, E), rm0 = ld(EC_UCON, 0, W);
  const S r0p = ld(EC_UCON, 0, No), r0m = ld(EC_UCON, 0, S_);
  const S mx00 = ld(EC_UCON, 1, n), mxp0 = ld(EC_UCON, 1, E), mxm0 = ld(EC_UCON, 1, W);
  const S my00 = ld(EC_UCON, 2, n), my0p = ld(EC_UCON, 2, No), my0m = ld(EC_UCON, 2, S_);
  const S E00 = ld(EC_UCON, 4, n);
  const S h_00 = eos_e(P, r00, p00) + p00 / r00;
  const S h_p0 = eos_e(P, rp0, pp0) + pp0 / rp0;
  const S h_m0 = eos_e(P, rm0, pm0) + pm0 / rm0;
  const S h_0p = eos_e(P, r0p, p0p) + p0p / r0p;
  const S h_0m = eos_e(P, r0m, p0m) + p0m / r0m;
  const S flux_xm = 0.5 * (h_m0 * mxm0 + h_00 * mx00);
  const S flux_xp = 0.5 * (h_00 * mx00 + h_p0 * mxp0);
  const S flux_ym = 0.5 * (h_0m * my0m + h_00 * my00);
  const S flux_yp = 0.5 * (h_00 * my00 + h_0p * my0p);
  out[0] = E00 - h / (P.dx) * (flux_xp - flux_xm) - h / (P.dy) * (flux_yp - flux_ym);
}

// ---- corner EMF: CT_CornerAssemble (constrained_transport.cpp:147-164) of the face EMFs
// ep0 = sx fx, e0p = sy fy and the cell EMF vy Bx - vx By of u_con (ct_flux.cpp:165-168)
enum { CC_FX = 0, CC_FY = 1, CC_UCON = 2 };
template <class S, class Ld>
__device__ __forceinline__ S cell_ez(Ld& ld, long long m) {
  const S r = ld(CC_UCON, 0, m);
  return ld(CC_UCON, 2, m) / r * ld(CC_UCON, 5, m) - ld(CC_UCON, 1, m) / r * ld(CC_UCON, 6, m);
}
// bnb: the neighbourhood Ez_bar is evaluated on.  It is nb itself except at a corner on
// x = x_0 or y = y_0 of a transmissive direction, where bound_cond_array has replaced
// Ez_bar by its value at the nearest interior corner (constrained_transport.cpp:150-155)
// while the correction terms still read the corner's own neighbourhood.
template <class S, class Ld>
__device__ __forceinline__ void ct_corner_at(const DevParams& P, double sx, double sy, const long long* nb,
                                             const long long* bnb, Ld& ld, S* out) {
  const long long c00 = nb[NB_C], c10 = nb[NB_E], c01 = nb[NB_N], c11 = nb[NB_NE];
  const double dx = P.dx, dy = P.dy;
  const S Ep0_00 = sx * ld(CC_FX, 0, c00), Ep0_01 = sx * ld(CC_FX, 0, c01);
  const S E0p_00 = sy * ld(CC_FY, 0, c00), E0p_10 = sy * ld(CC_FY, 0, c10);
  const S Et00 = cell_ez<S>(ld, c00), Et10 = cell_ez<S>(ld, c10), Et01 = cell_ez<S>(ld, c01), Et11 = cell_ez<S>(ld, c11);
  const S bar = 0.25 * (sx * ld(CC_FX, 0, bnb[NB_C]) + sx * ld(CC_FX, 0, bnb[NB_N]) + sy * ld(CC_FY, 0, bnb[NB_C]) +
                        sy * ld(CC_FY, 0, bnb[NB_E]));
  const S t1 = 0.5 * ((Ep0_00 - Et00) / (dx / 2.0) + (Ep0_01 - Et01) / (dx / 2.0));
  const S t2 = 0.5 * ((Et10 - Ep0_00) / (dx / 2.0) + (Et11 - Ep0_01) / (dx / 2.0));
  const S t3 = 0.5 * ((E0p_00 - Et00) / (dy / 2.0) + (E0p_10 - Et10) / (dy / 2.0));
  const S t4 = 0.5 * ((Et01 - E0p_00) / (dy / 2.0) + (Et11 - E0p_10) / (dy / 2.0));
  out[0] = bar + dx / 8.0 * (t1 - t2) + dy / 8.0 * (t3 - t4);
}
template <class S, class Ld>
__device__ __forceinline__ void ct_corner_cell(const DevParams& P, double sx, double sy, const long long* nb, Ld& ld,
                                               S* out) {
  ct_corner_at<S>(P, sx, sy, nb, nb, ld, out);
}

// ---- frozen pressure-operator coefficient hh = h(Qe) rho_e / rho (imex_subsystems.cpp:92-104)
// and the pressure p(Qe) of the stage combination
enum { HH_QE = 0, HH_UCON = 1 };
template <class S, class Ld>
__device__ __forceinline__ void hh_cell(const DevParams& P, const long long* nb, Ld& ld, S* out) {
  const long long n = nb[NB_C];
  S c[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) c[k] = ld(HH_QE, k, n);
  out[0] = calenthalpy(P, c) * c[0] / ld(HH_UCON, 0, n);
}
template <class S, class Ld>
__device__ __forceinline__ void pe_cell(const DevParams& P, const long long* nb, Ld& ld, S* out) {
  const long long n = nb[NB_C];
  S c[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) c[k] = ld(0, k, n);
  out[0] = pressure_of(P, c);
}

}  // namespace imex
