/* CPU restatement of one IMEX-RK time step of the reference 2D ideal-MHD solver.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle); see imex_oracle.h.  Every function
 * cites the reference file:line it restates.  Arithmetic follows the
 * reference expression by expression (same operand order, no FMA
 * contraction: built with -ffp-contract=off), so explicit sub-steps agree
 * with the reference bit for bit; implicit solves agree to solver tolerance
 * because reductions are summed serially in index order here.
 *
 * Periodic and transmissive boundaries (per direction, ora_set_bc): ghost cells
 * are replaced by index maps.  Periodic wraps, which reproduces the reference's
 * periodic ghost fills (boundary.cpp:46,118, timestep.cpp:184,213,
 * constrained_transport.cpp:13,32) exactly.  Transmissive clamps to the nearest
 * interior cell, which is what bound_cond_u, bound_cond_array, M_P / M_B and the
 * operators' max/min neighbour indices do for x_Transmissive / y_Transmissive
 * (boundary.cpp:7-16, timestep.cpp:168-175,195-204, implicit_operators.cpp:12-14,
 * 150-153).  Two things are not a clamp there and are restated explicitly:
 *   - the boundary normal faces (Bx at x = x_0, By at y = y_0) are degrees of
 *     freedom that CT evolves (constrained_transport.cpp:5-30); every face array
 *     carries them after its nx*ny interior values (bx: ny values, by: nx values);
 *   - the corner EMF at x_0 / y_0: its averaged part Ez_bar is clamped by
 *     bound_cond_array while its correction terms are evaluated at the boundary
 *     corner itself (constrained_transport.cpp:147-164).
 */
#include "imex_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { EnergyFormula = 0, PressureFormula = 1 };
enum { StaggerCT = 0, UnStaggerCT = 1, PotentialA = 2, NoDivFree = 3 };
enum { NoRecon = 0, Minmod = 1, VanLeer = 2, ENO3 = 3, WENO5 = 4 };
enum { PrimState = 0, ConsState = 1 };
enum { Fullydt = 0, Alfvendt = 1, IMEXdt = 2 };
enum { MaterialSpeedp = 0, AlfvenSpeedp = 1, Noaddvisp = 2 };
enum { ConservationofU = 0, DefinitionofU = 1 };
enum { no_correction = 0, once_correction = 1, all_correction = 2 };
enum { IDEAL_GAS = 0, REDLICH_KWONG = 1 };
enum { SUB_COMBINE = 0, SUB_CONVECTIVE, SUB_MAGNETIC, SUB_PFLUX, SUB_PRESSURE, SUB_CT, NSUB };
#define MAXRK 3
#define JMAX 25
#define EOS_NEWTON_CAP 200

typedef struct {
  int valid;
  double *u_con, *Qe, *Qs, *bx, *by, *bxQs, *byQs, *A, *A_s, *Fx, *Fy;
} snap_t;

static struct {
  int ready, nx, ny, R;
  int xclamp, yclamp; /* transmissive (clamped) directions; periodic otherwise */
  size_t N, NF;       /* cells; entries of a face array (N + nx + ny) */
  ora_params P;
  double dx, dy;
  double *prim, *cons, *cons_n, *Qe, *Qs, *wxL, *wxR, *wyL, *wyR;
  double *bx, *by, *bx_n, *by_n, *bxQe, *byQe, *bxQs, *byQs, *Fx, *Fy;
  double *A, *A_s, *A_e, *A_snap, *Hs, *HsA, *HsB, *Bsave;
  double Ae[MAXRK][MAXRK], Ai[MAXRK][MAXRK];
  double t, dt, adt, B_max_x, B_max_y, vx_max, vy_max, v_max, a_max, ch, ch_x, ch_y;
  double cA_x, cA_y, cA, prev_dt, Mbig, min_p_ever;
  int timestep, max_floored, snap_on;
  snap_t snaps[MAXRK][NSUB];
} G;

/* ------------------------------------------------------------------ */
/* indexing                                                           */
/* ------------------------------------------------------------------ */
static inline int CI(int i) {
  int nx = G.nx;
  if (G.xclamp) return i < 0 ? 0 : (i >= nx ? nx - 1 : i);
  i %= nx;
  return i < 0 ? i + nx : i;
}
static inline int CJ(int j) {
  int ny = G.ny;
  if (G.yclamp) return j < 0 ? 0 : (j >= ny ? ny - 1 : j);
  j %= ny;
  return j < 0 ? j + ny : j;
}
static inline size_t ID(int i, int j) { return (size_t)CI(i) + (size_t)G.nx * (size_t)CJ(j); }
/* x-face (i+1/2, j) and y-face (i, j+1/2) of a face array: left of x_0 / below y_0 a
 * transmissive direction reads the boundary face (bound_cond_staggered's normal rule) */
static inline double BXF(const double* a, int i, int j) {
  return (i < 0 && G.xclamp) ? a[G.N + (size_t)CJ(j)] : a[ID(i, j)];
}
static inline double BYF(const double* a, int i, int j) {
  return (j < 0 && G.yclamp) ? a[G.N + (size_t)CI(i)] : a[ID(i, j)];
}
/* a plane of A (or of the A-form operator's vector) with the ghosts of bound_cond_A,
 * boundary.cpp:177-292: a transmissive direction extrapolates linearly from its two nearest
 * interior cells, x first and then y on the x-extrapolated rows; a periodic one wraps */
static double agh_row(const double* a, int i, int j) {
  const int nx = G.nx;
  const double* r = a + (size_t)nx * (size_t)j;
  if (G.xclamp && i < 0) {
    double slope = r[1] - r[0];
    return r[0] - (double)(-i) * slope;
  }
  if (G.xclamp && i >= nx) {
    double slope = r[nx - 1] - r[nx - 2];
    return r[nx - 1] + (double)(i - nx + 1) * slope;
  }
  return r[CI(i)];
}
static double agh(const double* a, int i, int j) {
  const int ny = G.ny;
  if (G.yclamp && j < 0) {
    double a0 = agh_row(a, i, 0), slope = agh_row(a, i, 1) - a0;
    return a0 - (double)(-j) * slope;
  }
  if (G.yclamp && j >= ny) {
    double aT = agh_row(a, i, ny - 1), slope = aT - agh_row(a, i, ny - 2);
    return aT + (double)(j - ny + 1) * slope;
  }
  return agh_row(a, i, CJ(j));
}
#define PL(a, k) ((a) + (size_t)(k)*G.N)
#define AT(a, k, i, j) ((a)[(size_t)(k)*G.N + ID(i, j)])

static void load8(const double* a, size_t idx, double o[8]) {
  for (int k = 0; k < 8; ++k) o[k] = a[(size_t)k * G.N + idx];
}
static double* alloc(size_t n) {
  double* p = (double*)calloc(n, sizeof(double));
  return p;
}

/* ------------------------------------------------------------------ */
/* EOS, config.hpp:130-239                                            */
/* ------------------------------------------------------------------ */
#define PP G.P
static double rk_fT(double T, double v, double p) { return PP.m_R * T / (v - PP.m_b) - PP.m_alfa / sqrt(T) / v / (v + PP.m_b) - p; }
static double rk_dfT(double T, double v) { return PP.m_R / (v - PP.m_b) + 0.5 * PP.m_alfa / T / sqrt(T) / v / (v + PP.m_b); }
static double rk_fp(double T, double v, double e) {
  double U = log(v / (v + PP.m_b));
  return PP.m_cv * T + 1.5 * PP.m_alfa / PP.m_b * U / sqrt(T) - e;
}
static double rk_dfp(double T, double v) {
  double U = log(v / (v + PP.m_b));
  return PP.m_cv - 0.75 * PP.m_alfa / PP.m_b * U / T / sqrt(T);
}
/* config.hpp:137-144 (iteration cap added; the reference loops until converged) */
static double rk_T_from_rho_p(double rho, double p) {
  double v = 1.0 / rho;
  double T_old, T_new = (1.0 / rho - PP.m_b) * (p + PP.m_alfa * rho * rho) / PP.m_R;
  int it = 0;
  do {
    T_old = T_new;
    T_new = T_old - rk_fT(T_old, v, p) / rk_dfT(T_old, v);
  } while (fabs(T_new - T_old) / fabs(T_old) > 1e-14 && ++it < EOS_NEWTON_CAP);
  return T_new;
}
/* config.hpp:146-151 */
static double rk_e_from_rho_p(double rho, double p) {
  double v = 1.0 / rho;
  double T = rk_T_from_rho_p(rho, p);
  double U = log(v / (v + PP.m_b));
  return PP.m_cv * T + 1.5 * PP.m_alfa / PP.m_b * U / sqrt(T);
}
/* config.hpp:153-161 */
static double rk_p_from_rho_e(double rho, double e) {
  double v = 1.0 / rho;
  double T_old, T_new = (e + rho * PP.m_alfa) / PP.m_cv;
  int it = 0;
  do {
    T_old = T_new;
    T_new = T_old - rk_fp(T_old, v, e) / rk_dfp(T_old, v);
  } while (fabs(T_new - T_old) / fabs(T_old) > 1e-14 && ++it < EOS_NEWTON_CAP);
  double a = PP.m_alfa / sqrt(T_new);
  return PP.m_R * T_new / (v - PP.m_b) - a / v / (v + PP.m_b);
}
/* config.hpp:163-173 */
static double rk_sound(double rho, double p) {
  double v = 1.0 / rho;
  double T = rk_T_from_rho_p(rho, p);
  double U = log(v / (v + PP.m_b));
  double p_T = PP.m_R / (v - PP.m_b) + PP.m_alfa / (2.0 * T * sqrt(T) * v * (v + PP.m_b));
  double e_T = PP.m_cv - 0.75 * PP.m_alfa / PP.m_b * U / (T * sqrt(T));
  double vmb = v - PP.m_b, vpb = v + PP.m_b;
  double p_v = -PP.m_R * T / (vmb * vmb) + PP.m_alfa * (2.0 * v + PP.m_b) / (sqrt(T) * v * v * (vpb * vpb));
  double e_v = 1.5 * PP.m_alfa / PP.m_b * (1.0 / v - 1.0 / (v + PP.m_b)) / sqrt(T);
  double a2 = p / (rho * rho) * (p_T / e_T) + v * v * (e_v - e_T * (p_v / p_T));
  return sqrt(a2);
}
static double eos_p(double rho, double e) {
  return PP.eos_type == IDEAL_GAS ? (PP.gamma_plasma - 1.0) * rho * e : rk_p_from_rho_e(rho, e);
}
static double eos_e(double rho, double p) {
  return PP.eos_type == IDEAL_GAS ? p / ((PP.gamma_plasma - 1.0) * rho) : rk_e_from_rho_p(rho, p);
}
static double eos_a(double rho, double p) {
  return PP.eos_type == IDEAL_GAS ? sqrt(PP.gamma_plasma * p / rho) : rk_sound(rho, p);
}
static double eos_a2(double rho, double p) {
  double a = eos_a(rho, p);
  return a * a;
}
/* config.hpp:192-198 */
static double eos_fast(double rho, double p, double Bn, double B2) {
  double a2 = eos_a2(rho, p);
  double t = a2 + B2 / rho;
  double disc = t * t - 4.0 * a2 * Bn * Bn / rho;
  if (disc < 0) disc = 0;
  return sqrt(0.5 * (t + sqrt(disc)));
}
/* config.hpp:206-239 */
static double Vbase(double p, double rho) {
  return PP.eos_type == IDEAL_GAS ? p / (PP.gamma_plasma - 1.0) : rho * rk_e_from_rho_p(rho, p);
}
static double Vbase_slope(double p, double rho) {
  if (PP.eos_type == IDEAL_GAS) return 1.0 / (PP.gamma_plasma - 1.0);
  const double d = 1e-8;
  double ep = rk_e_from_rho_p(rho, p + d);
  double em = rk_e_from_rho_p(rho, p - d);
  return rho * (ep - em) / (2.0 * d);
}
static double V_mod(double p, double rho) {
  if (!PP.floor_on) return Vbase(p, rho);
  return (p >= PP.p_floor) ? Vbase(p, rho) : Vbase(PP.p_floor, rho) + G.Mbig * (p - PP.p_floor);
}
static double V_slope(double p, double rho) {
  if (!PP.floor_on) return Vbase_slope(p, rho);
  return (p >= PP.p_floor) ? Vbase_slope(p, rho) : G.Mbig;
}

/* ------------------------------------------------------------------ */
/* pointwise state functions, state.cpp / reconstruction.cpp / timestep.cpp */
/* ------------------------------------------------------------------ */
/* reconstruction.cpp:291-304 */
static double calecon(const double* c) {
  double rho = c[0], vx = c[1] / c[0], vy = c[2] / c[0], vz = c[3] / c[0];
  double U = c[4], Bx = c[5], By = c[6], Bz = c[7];
  double B2 = Bx * Bx + By * By + Bz * Bz;
  double v2 = vx * vx + vy * vy + vz * vz;
  return (U - 0.5 * rho * v2 - 0.5 * B2) / rho;
}
/* state.cpp:206-218 */
static void con2pri(double* pri, const double* con) {
  double e = calecon(con);
  pri[0] = con[0];
  pri[1] = con[1] / con[0];
  pri[2] = con[2] / con[0];
  pri[3] = con[3] / con[0];
  pri[4] = eos_p(con[0], e);
  pri[5] = con[5];
  pri[6] = con[6];
  pri[7] = con[7];
}
/* state.cpp:220-240 */
static void pri2con(double* con, const double* pri) {
  double e = eos_e(pri[0], pri[4]);
  double vx = pri[1], vy = pri[2], vz = pri[3], Bx = pri[5], By = pri[6], Bz = pri[7];
  double B2 = Bx * Bx + By * By + Bz * Bz;
  double v2 = vx * vx + vy * vy + vz * vz;
  double r = pri[0];
  con[0] = r;
  con[1] = r * pri[1];
  con[2] = r * pri[2];
  con[3] = r * pri[3];
  con[4] = r * e + 0.5 * r * v2 + 0.5 * B2;
  con[5] = pri[5];
  con[6] = pri[6];
  con[7] = pri[7];
}
static void grid_con2pri(double* pri, const double* con) {
  double c[8], p[8];
  for (size_t n = 0; n < G.N; ++n) {
    load8(con, n, c);
    con2pri(p, c);
    for (int k = 0; k < 8; ++k) pri[(size_t)k * G.N + n] = p[k];
  }
}
static void grid_pri2con(double* con, const double* pri) {
  double c[8], p[8];
  for (size_t n = 0; n < G.N; ++n) {
    load8(pri, n, p);
    pri2con(c, p);
    for (int k = 0; k < 8; ++k) con[(size_t)k * G.N + n] = c[k];
  }
}
/* timestep.cpp:239-247 */
static double calkinetic(const double* c) {
  double rho = c[0], vx = c[1] / c[0], vy = c[2] / c[0], vz = c[3] / c[0];
  return 0.5 * rho * (vx * vx + vy * vy + vz * vz);
}
/* timestep.cpp:224-230 */
static double calenthalpy(const double* c) {
  double e = calecon(c);
  double pri[8];
  con2pri(pri, c);
  return e + pri[4] / pri[0];
}

/* ------------------------------------------------------------------ */
/* reconstruction, reconstruction.cpp:5-287                           */
/* ------------------------------------------------------------------ */
static void recon_1d(int scheme, double um2, double um1, double u0, double up1, double up2, double* wL,
                     double* wR, int vortex_central) {
  double sR = up1 - u0, sL = u0 - um1, c = 0.0;
  switch (scheme) {
    case NoRecon:
      *wL = u0;
      *wR = u0;
      break;
    case Minmod: /* reconstruction.cpp:46-75 */
      if (sL * sR <= 0) c = 0;
      else if (fabs(sR) <= fabs(sL)) c = sR;
      else if (fabs(sL) < fabs(sR)) c = sL;
      if (vortex_central) c = 0.5 * (sL + sR);
      *wL = u0 - 0.5 * c;
      *wR = u0 + 0.5 * c;
      break;
    case VanLeer: /* reconstruction.cpp:76-103 */
      if (fabs(sR) < 1e-16) c = 0;
      else {
        double r = sL / sR;
        if (r < 0) c = 0;
        else c = fmin(2 / (1 + r), (2 * r) / (1 + r));
      }
      *wL = u0 - 0.5 * c * sL;
      *wR = u0 + 0.5 * c * sR;
      break;
    case ENO3: { /* reconstruction.cpp:104-143 */
      double q0L = -1.0 / 6.0 * um2 + 5.0 / 6.0 * um1 + 1.0 / 3.0 * u0;
      double q1L = 1.0 / 3.0 * um1 + 5.0 / 6.0 * u0 - 1.0 / 6.0 * up1;
      double q2L = 11.0 / 6.0 * u0 - 7.0 / 6.0 * up1 + 1.0 / 3.0 * up2;
      double q0R = 1.0 / 3.0 * um2 - 7.0 / 6.0 * um1 + 11.0 / 6.0 * u0;
      double q1R = -1.0 / 6.0 * um1 + 5.0 / 6.0 * u0 + 1.0 / 3.0 * up1;
      double q2R = 1.0 / 3.0 * u0 + 5.0 / 6.0 * up1 - 1.0 / 6.0 * up2;
      double d1 = fabs(u0 - um1), d2 = fabs(up1 - u0), d3, d4;
      if (d1 >= d2) {
        d3 = fabs(fabs(up2 - up1) - fabs(up1 - u0));
        d4 = fabs(fabs(up1 - u0) - fabs(u0 - um1));
        if (d3 >= d4) { *wL = q1L; *wR = q1R; }
        else { *wL = q2L; *wR = q2R; }
      } else {
        d3 = fabs(fabs(u0 - um1) - fabs(um1 - um2));
        d4 = fabs(fabs(up1 - u0) - fabs(u0 - um1));
        if (d4 >= d3) { *wL = q0L; *wR = q0R; }
        else { *wL = q1L; *wR = q1R; }
      }
      break;
    }
    case WENO5: { /* reconstruction.cpp:184-224 */
      double a0 = um2 - 2 * um1 + u0, b0 = um2 - 4 * um1 + 3 * u0;
      double a1 = um1 - 2 * u0 + up1, b1 = um1 - up1;
      double a2 = u0 - 2 * up1 + up2, b2 = 3 * u0 - 4 * up1 + up2;
      double beta0 = 13.0 / 12.0 * (a0 * a0) + 1.0 / 4.0 * (b0 * b0);
      double beta1 = 13.0 / 12.0 * (a1 * a1) + 1.0 / 4.0 * (b1 * b1);
      double beta2 = 13.0 / 12.0 * (a2 * a2) + 1.0 / 4.0 * (b2 * b2);
      double e0 = 1e-6 + beta0, e1 = 1e-6 + beta1, e2 = 1e-6 + beta2;
      double q0 = -1.0 / 6.0 * um2 + 5.0 / 6.0 * um1 + 1.0 / 3.0 * u0;
      double q1 = 1.0 / 3.0 * um1 + 5.0 / 6.0 * u0 - 1.0 / 6.0 * up1;
      double q2 = 11.0 / 6.0 * u0 - 7.0 / 6.0 * up1 + 1.0 / 3.0 * up2;
      double w0b = 3.0 / 10.0 / (e0 * e0), w1b = 6.0 / 10.0 / (e1 * e1), w2b = 1.0 / 10.0 / (e2 * e2);
      double w0 = w0b / (w0b + w1b + w2b), w1 = w1b / (w0b + w1b + w2b), w2 = w2b / (w0b + w1b + w2b);
      *wL = w0 * q0 + w1 * q1 + w2 * q2;
      q0 = 1.0 / 3.0 * um2 - 7.0 / 6.0 * um1 + 11.0 / 6.0 * u0;
      q1 = -1.0 / 6.0 * um1 + 5.0 / 6.0 * u0 + 1.0 / 3.0 * up1;
      q2 = 1.0 / 3.0 * u0 + 5.0 / 6.0 * up1 - 1.0 / 6.0 * up2;
      w0b = 1.0 / 10.0 / (e0 * e0);
      w1b = 6.0 / 10.0 / (e1 * e1);
      w2b = 3.0 / 10.0 / (e2 * e2);
      w0 = w0b / (w0b + w1b + w2b);
      w1 = w1b / (w0b + w1b + w2b);
      w2 = w2b / (w0b + w1b + w2b);
      *wR = w0 * q0 + w1 * q1 + w2 * q2;
      break;
    }
  }
}

/* TVDReconstruction: w_xL, w_xR, w_yL, w_yR of grid Q (8 planes each) */
static void reconstruct(const double* Q, double* wxL, double* wxR, double* wyL, double* wyR) {
  const double* u = Q;
  double* tmp = NULL;
  if (PP.reconstate == PrimState) {
    tmp = alloc(8 * G.N);
    grid_con2pri(tmp, Q);
    u = tmp;
  }
  for (int k = 0; k < 8; ++k) {
    const double* a = PL(u, k);
    for (int j = 0; j < G.ny; ++j)
      for (int i = 0; i < G.nx; ++i) {
        size_t o = (size_t)k * G.N + ID(i, j);
        /* x direction: the vortex special case never reaches x (c is overwritten), y only */
        recon_1d(PP.recon, a[ID(i - 2, j)], a[ID(i - 1, j)], a[ID(i, j)], a[ID(i + 1, j)], a[ID(i + 2, j)],
                 &wxL[o], &wxR[o], 0);
        recon_1d(PP.recon, a[ID(i, j - 2)], a[ID(i, j - 1)], a[ID(i, j)], a[ID(i, j + 1)], a[ID(i, j + 2)],
                 &wyL[o], &wyR[o], PP.recon == Minmod && PP.vortex_test);
      }
  }
  if (tmp) {
    double* ws[4] = {wxL, wxR, wyL, wyR};
    for (int q = 0; q < 4; ++q) {
      memcpy(tmp, ws[q], 8 * G.N * sizeof(double));
      grid_pri2con(ws[q], tmp);
    }
    free(tmp);
  }
}

/* ------------------------------------------------------------------ */
/* explicit fluxes, flux.cpp / state.cpp                              */
/* ------------------------------------------------------------------ */
/* state.cpp:27-44 / 86-106 */
static void f_conv(double* f, const double* c, int dir) {
  double rho = c[0], vx = c[1] / c[0], vy = c[2] / c[0], vz = c[3] / c[0];
  double k = calkinetic(c);
  double vn = dir == 0 ? vx : vy;
  f[0] = rho * vn;
  f[1] = rho * vx * vn;
  f[2] = rho * vy * vn;
  f[3] = rho * vz * vn;
  f[4] = k * vn;
}
static double smax_of(const double* QL, const double* QR, int dir) {
  if (PP.GLF) return G.a_max;
  return fmax(fabs(QL[1 + dir] / QL[0]), fabs(QR[1 + dir] / QR[0]));
}
/* flux.cpp:329-406 RusanovC_x / RusanovC_y */
static void rusanovC(const double* QL, const double* QR, double* F, int dir) {
  double fL[5], fR[5];
  f_conv(fL, QL, dir);
  f_conv(fR, QR, dir);
  if (PP.formula == EnergyFormula) fL[4] = fR[4] = 0;
  double s = smax_of(QL, QR, dir);
  for (int k = 0; k < 5; ++k) F[k] = 0.5 * (fL[k] + fR[k]) - 0.5 * s * (QR[k] - QL[k]);
}
/* state.cpp:298-322 MagneticFlux_Pressure_x/y */
static void magflux_p(double* f, const double* Q, int dir) {
  double B2 = Q[5] * Q[5] + Q[6] * Q[6] + Q[7] * Q[7];
  double vB = (Q[1] * Q[5] + Q[2] * Q[6] + Q[3] * Q[7]) / Q[0];
  f[0] = 0;
  if (dir == 0) {
    f[1] = B2 * 0.5 - Q[5] * Q[5];
    f[2] = -Q[5] * Q[6];
    f[3] = -Q[5] * Q[7];
    f[4] = Q[1] / Q[0] * B2 - Q[5] * vB;
  } else {
    f[1] = -Q[5] * Q[6];
    f[2] = B2 * 0.5 - Q[6] * Q[6];
    f[3] = -Q[6] * Q[7];
    f[4] = Q[2] / Q[0] * B2 - Q[6] * vB;
  }
}
/* flux.cpp:202-287 Pressure_flux_x / Pressure_flux_y */
static void pressure_flux(const double* QL, const double* QR, double* F, int dir) {
  double fC[5], fB[5], fL[5], fR[5];
  f_conv(fC, QL, dir);
  magflux_p(fB, QL, dir);
  for (int k = 0; k < 5; ++k) fL[k] = fC[k] + fB[k];
  f_conv(fC, QR, dir);
  magflux_p(fB, QR, dir);
  for (int k = 0; k < 5; ++k) fR[k] = fC[k] + fB[k];
  double s = smax_of(QL, QR, dir);
  for (int k = 0; k < 5; ++k) F[k] = 0.5 * (fL[k] + fR[k]) - 0.5 * s * (QR[k] - QL[k]);
}
/* state.cpp:272-296 MagneticFlux_x/y (energy formula) */
static void magflux_e(double* f, const double* Q, int dir) {
  const double g = PP.gamma_plasma;
  double B2 = Q[5] * Q[5] + Q[6] * Q[6] + Q[7] * Q[7];
  double vB = (Q[1] * Q[5] + Q[2] * Q[6] + Q[3] * Q[7]) / Q[0];
  f[0] = 0;
  if (dir == 0) {
    f[1] = (2 - g) * B2 * 0.5 - Q[5] * Q[5];
    f[2] = -Q[5] * Q[6];
    f[3] = -Q[5] * Q[7];
    f[4] = Q[1] / Q[0] * B2 * 0.5 - Q[5] * vB;
  } else {
    f[1] = -Q[5] * Q[6];
    f[2] = (2 - g) * B2 * 0.5 - Q[6] * Q[6];
    f[3] = -Q[6] * Q[7];
    f[4] = Q[2] / Q[0] * B2 * 0.5 - Q[6] * vB;
  }
}
/* flux.cpp:78-161 Energy_flux_x / Energy_flux_y: convective (energy slot zeroed) +
   magnetic + kinetic-energy flux f/g_KineticEnergyFlux (state.cpp:325-345) */
static void energy_flux(const double* QL, const double* QR, double* F, int dir) {
  double fC[5], fB[5], fK[5], fL[5], fR[5];
  const double* Q[2] = {QL, QR};
  double* out[2] = {fL, fR};
  for (int s = 0; s < 2; ++s) {
    f_conv(fC, Q[s], dir);
    fC[4] = 0;
    magflux_e(fB, Q[s], dir);
    for (int k = 0; k < 5; ++k) fK[k] = 0;
    fK[1 + dir] = -(PP.gamma_plasma - 1) * 0.5 * (Q[s][1] * Q[s][1] + Q[s][2] * Q[s][2] + Q[s][3] * Q[s][3]) / Q[s][0];
    for (int k = 0; k < 5; ++k) out[s][k] = fC[k] + fB[k] + fK[k];
  }
  double s = smax_of(QL, QR, dir);
  for (int k = 0; k < 5; ++k) F[k] = 0.5 * (fL[k] + fR[k]) - 0.5 * s * (QR[k] - QL[k]);
}
typedef void (*flux_fn)(const double*, const double*, double*, int);

/* flux.cpp:409-455 / 290-326: u_con[0..4] = Qs - h/dx (fp - fm) - h/dy (gp - gm) */
static void flux_update(flux_fn fn, double* ucon, const double* Qs, const double* wxL, const double* wxR,
                        const double* wyL, const double* wyR, double h) {
  double QL[8], QR[8], fp[5], fm[5], gp[5], gm[5];
  for (int j = 0; j < G.ny; ++j)
    for (int i = 0; i < G.nx; ++i) {
      load8(wxR, ID(i, j), QL);
      load8(wxL, ID(i + 1, j), QR);
      fn(QL, QR, fp, 0);
      load8(wyR, ID(i, j), QL);
      load8(wyL, ID(i, j + 1), QR);
      fn(QL, QR, gp, 1);
      load8(wxR, ID(i - 1, j), QL);
      load8(wxL, ID(i, j), QR);
      fn(QL, QR, fm, 0);
      load8(wyR, ID(i, j - 1), QL);
      load8(wyL, ID(i, j), QR);
      fn(QL, QR, gm, 1);
      size_t o = ID(i, j);
      for (int k = 0; k < 5; ++k)
        ucon[(size_t)k * G.N + o] = Qs[(size_t)k * G.N + o] - h / G.dx * (fp[k] - fm[k]) - h / G.dy * (gp[k] - gm[k]);
    }
}

/* ------------------------------------------------------------------ */
/* shock detector, flux.cpp:5-76                                      */
/* ------------------------------------------------------------------ */
static void shock_detector(double* eta, const double* Q) {
  double* pri = alloc(8 * G.N);
  double* chit = alloc(G.N);
  grid_con2pri(pri, Q);
  double h = G.dx < G.dy ? G.dx : G.dy; /* std::min(dx, dy) */
  for (int i = 0; i < G.nx; ++i)
    for (int j = 0; j < G.ny; ++j) {
      double cfmin = 1.0e300;
      for (int di = -1; di <= 1; di++)
        for (int dj = -1; dj <= 1; dj++) {
          size_t n = ID(i + di, j + dj);
          double rho = pri[n], p = pri[4 * G.N + n], bx = pri[5 * G.N + n], by = pri[6 * G.N + n],
                 bz = pri[7 * G.N + n];
          double a2 = eos_a2(rho, p);
          double cA2 = (bx * bx + by * by + bz * bz) / rho;
          double cf = sqrt(a2 + cA2);
          if (cf < cfmin) cfmin = cf;
        }
      double div_u = (AT(pri, 1, i + 1, j) - AT(pri, 1, i - 1, j)) / (2.0 * G.dx) +
                     (AT(pri, 2, i, j + 1) - AT(pri, 2, i, j - 1)) / (2.0 * G.dy);
      double num = h * div_u + PP.shock_kappa1 * cfmin;
      double den = PP.shock_kappa1 * cfmin;
      double q = -num / den;
      double mx = (0.0 < q) ? q : 0.0;      /* std::max(0.0, q) */
      chit[ID(i, j)] = (mx < 1.0) ? mx : 1.0; /* std::min(1.0, mx) */
    }
  for (int i = 0; i < G.nx; ++i)
    for (int j = 0; j < G.ny; ++j) {
      double m = 0.0;
      for (int di = -1; di <= 1; di++)
        for (int dj = -1; dj <= 1; dj++)
          if (chit[ID(i + di, j + dj)] > m) m = chit[ID(i + di, j + dj)];
      eta[ID(i, j)] = m;
    }
  free(pri);
  free(chit);
}

/* ------------------------------------------------------------------ */
/* GMRES, implicit_operators.cpp:793-919                              */
/* ------------------------------------------------------------------ */
typedef void (*op_fn)(const double* x, double* Ax);
typedef void (*pc_fn)(const double* in, double* out);

static double dotv(const double* a, const double* b, int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

static void gmres(double* x, const double* b, op_fn A, pc_fn M, int dim) {
  const int outmax = dim;
  double** v = (double**)malloc((JMAX + 1) * sizeof(double*));
  double** Av = (double**)malloc((JMAX + 1) * sizeof(double*));
  for (int i = 0; i <= JMAX; ++i) {
    v[i] = alloc(dim);
    Av[i] = alloc(dim);
  }
  double *w = alloc(dim), *Ax = alloc(dim), *r0 = alloc(dim), *tmp = alloc(dim);
  double H[JMAX + 2][JMAX + 2], alpha[JMAX + 2], gam[JMAX + 2], s[JMAX + 2], c[JMAX + 2];
  memset(alpha, 0, sizeof alpha);
  memset(gam, 0, sizeof gam);
  memset(s, 0, sizeof s);
  memset(c, 0, sizeof c);
  double tol_eff = PP.GMREStol;
  for (int outer = 0; outer < outmax; outer++) {
    A(x, Ax);
    for (int i = 0; i < dim; ++i) tmp[i] = b[i] - Ax[i];
    if (M) M(tmp, r0);
    else memcpy(r0, tmp, dim * sizeof(double));
    gam[0] = sqrt(dotv(r0, r0, dim));
    if (outer == 0) tol_eff = PP.GMREStol * gam[0] + PP.GMREStol;
    if (gam[0] <= tol_eff) goto done;
    for (int i = 0; i < dim; ++i) v[0][i] = r0[i] / gam[0];
    A(v[0], Ax);
    if (M) M(Ax, Av[0]);
    else memcpy(Av[0], Ax, dim * sizeof(double));
    memset(H, 0, sizeof H);
    for (int j = 0; j < JMAX; j++) {
      for (int i = 0; i <= j; i++) H[i][j] = dotv(v[i], Av[j], dim);
      memcpy(w, Av[j], dim * sizeof(double));
      for (int i = 0; i <= j; i++)
        for (int n = 0; n < dim; ++n) w[n] = w[n] - H[i][j] * v[i][n];
      H[j + 1][j] = sqrt(dotv(w, w, dim));
      for (int i = 0; i < j; i++) {
        double t1 = c[i + 1] * H[i][j] + s[i + 1] * H[i + 1][j];
        double t2 = s[i + 1] * H[i][j] - c[i + 1] * H[i + 1][j];
        H[i][j] = t1;
        H[i + 1][j] = t2;
      }
      double beta = sqrt(H[j][j] * H[j][j] + H[j + 1][j] * H[j + 1][j]);
      s[j + 1] = H[j + 1][j] / beta;
      c[j + 1] = H[j][j] / beta;
      H[j][j] = beta;
      gam[j + 1] = s[j + 1] * gam[j];
      gam[j] = c[j + 1] * gam[j];
      if (gam[j + 1] > tol_eff) {
        for (int n = 0; n < dim; ++n) v[j + 1][n] = w[n] / H[j + 1][j];
        A(v[j + 1], Ax);
        if (M) M(Ax, Av[j + 1]);
        else memcpy(Av[j + 1], Ax, dim * sizeof(double));
      } else {
        for (int i = j; i >= 0; i--) {
          alpha[i] = gam[i];
          for (int k = i + 1; k <= j; k++) alpha[i] -= H[i][k] * alpha[k];
          alpha[i] /= H[i][i];
        }
        for (int i = 0; i <= j; i++)
          for (int n = 0; n < dim; ++n) x[n] = x[n] + alpha[i] * v[i][n];
        goto done;
      }
    }
    memset(alpha, 0, sizeof alpha);
    for (int i = JMAX - 1; i >= 0; i--) {
      alpha[i] = gam[i];
      for (int k = i + 1; k < JMAX; k++) alpha[i] -= H[i][k] * alpha[k];
      alpha[i] /= H[i][i];
    }
    for (int i = 0; i < JMAX; i++)
      for (int n = 0; n < dim; ++n) x[n] = x[n] + alpha[i] * v[i][n];
  }
done:
  for (int i = 0; i <= JMAX; ++i) {
    free(v[i]);
    free(Av[i]);
  }
  free(v);
  free(Av);
  free(w);
  free(Ax);
  free(r0);
  free(tmp);
}

/* ------------------------------------------------------------------ */
/* operator context (frozen coefficients of the current solve)        */
/* ------------------------------------------------------------------ */
static struct {
  const double *ucon, *Qe, *Qs;
  double h;
  double *hh, *eta, *pe, *vscale, *tdiag, *pfreeze;
  int jac;
  double gmax_bx, gmax_by;
} OP;

/* Local Lax-Friedrichs speed of one cell for the magnetic viscosity (GLF = false):
   0.5 (|v| + sqrt(v^2 + 4 |B|^2 / rho)) of the primitive state of conserved state c along
   dir (implicit_operators.cpp:324-335 and 473-480, ct_flux.cpp:81-84 and 116-119) */
static double lf_speed(const double* c, int dir) {
  double rho = c[0], v = c[1 + dir] / c[0];
  return 0.5 * (fabs(v) + sqrt(v * v + 4.0 * (c[5] * c[5] + c[6] * c[6] + c[7] * c[7]) / rho));
}
static double lf_speed_at(const double* Q, int i, int j, int dir) {
  double c[8];
  load8(Q, ID(i, j), c);
  return lf_speed(c, dir);
}
/* the pressure viscosity's local speed of one cell (implicit_operators.cpp:587-598): |v_dir|
   (MaterialSpeedp), |B_dir| / sqrt(rho) (AlfvenSpeedp), 0 (Noaddvisp) */
static double pv_speed_at(const double* Q, int i, int j, int dir) {
  double c[8];
  load8(Q, ID(i, j), c);
  if (PP.add_pvisc == MaterialSpeedp) return fabs(c[1 + dir] / c[0]);
  if (PP.add_pvisc == AlfvenSpeedp) return fabs(c[5 + dir] / sqrt(c[0]));
  return 0.0;
}

/* enthalpy ratio h(Qe) rho_e / rho (implicit_operators.cpp:527-531) */
static double hhat_at(size_t n) {
  double c[8];
  load8(OP.Qe, n, c);
  return calenthalpy(c) * OP.Qe[n] / OP.ucon[n];
}

/* Pressure_Subsystem_AX, implicit_operators.cpp:505-616 (GLF, periodic) */
static void pressure_ax(const double* x, double* Ax) {
  const double h = OP.h, dx = G.dx, dy = G.dy;
  double nu_x = 0.0, nu_y = 0.0;
  if (PP.add_pvisc == MaterialSpeedp) {
    nu_x = G.vx_max * dx;
    nu_y = G.vy_max * dy;
  } else if (PP.add_pvisc == AlfvenSpeedp) {
    nu_x = G.cA_x * dx;
    nu_y = G.cA_y * dy;
  }
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      size_t c = ID(i, j), e = ID(i + 1, j), w = ID(i - 1, j), n = ID(i, j + 1), s = ID(i, j - 1);
      double h00 = OP.hh[c], hp0 = OP.hh[e], hm0 = OP.hh[w], h0p = OP.hh[n], h0m = OP.hh[s];
      double pii = x[c];
      double Vdiag = OP.jac ? V_slope(OP.pfreeze[c], OP.ucon[c]) : (1.0 / (PP.gamma_plasma - 1.0));
      double p_0m = x[s];
      double r = Vdiag * pii -
                 h * h *
                     (1 / (dx * dx) * (0.5 * (hp0 + h00) * (x[e] - x[c]) - 0.5 * (h00 + hm0) * (x[c] - x[w])) +
                      1 / (dy * dy) * (0.5 * (h0p + h00) * (x[n] - x[c]) - 0.5 * (h0m + h00) * (x[c] - p_0m)));
      const double* et = OP.eta;
      double lap_p;
      if (PP.GLF) {
        lap_p = nu_x / (dx * dx) *
                    (0.5 * (et[e] + et[c]) * (x[e] - pii) - 0.5 * (et[c] + et[w]) * (pii - x[w])) +
                nu_y / (dy * dy) *
                    (0.5 * (et[n] + et[c]) * (x[n] - pii) - 0.5 * (et[c] + et[s]) * (pii - x[s]));
      } else { /* implicit_operators.cpp:584-607 */
        double sx = pv_speed_at(OP.Qe, i, j, 0), sy = pv_speed_at(OP.Qe, i, j, 1);
        double nu_x_p = fmax(sx, pv_speed_at(OP.Qe, i + 1, j, 0)) * dx;
        double nu_x_m = fmax(sx, pv_speed_at(OP.Qe, i - 1, j, 0)) * dx;
        double nu_y_p = fmax(sy, pv_speed_at(OP.Qe, i, j + 1, 1)) * dy;
        double nu_y_m = fmax(sy, pv_speed_at(OP.Qe, i, j - 1, 1)) * dy;
        lap_p = 1 / (dx * dx) *
                    (0.5 * (et[e] + et[c]) * nu_x_p * (x[e] - pii) - 0.5 * (et[c] + et[w]) * nu_x_m * (pii - x[w])) +
                1 / (dy * dy) *
                    (0.5 * (et[n] + et[c]) * nu_y_p * (x[n] - pii) - 0.5 * (et[c] + et[s]) * nu_y_m * (pii - x[s]));
      }
      Ax[c] = r - OP.vscale[c] * h * lap_p;
    }
}
/* precP, implicit_operators.cpp:650-662 */
static void pressure_pc(const double* in, double* out) {
  const double a = 1.0 / (PP.gamma_plasma - 1.0);
  for (size_t n = 0; n < G.N; ++n) {
    double Vd = OP.jac ? V_slope(OP.pfreeze[n], OP.ucon[n]) : a;
    out[n] = in[n] / (Vd + OP.tdiag[n]);
  }
}
static void pressure_setup(const double* ucon, const double* Qe, const double* Qs, double h) {
  OP.ucon = ucon;
  OP.Qe = Qe;
  OP.Qs = Qs;
  OP.h = h;
  free(OP.hh); free(OP.eta); free(OP.pe); free(OP.vscale); free(OP.tdiag);
  OP.hh = alloc(G.N);
  OP.eta = alloc(G.N);
  OP.pe = alloc(G.N);
  OP.vscale = alloc(G.N);
  OP.tdiag = alloc(G.N);
  double c[8], p[8];
  for (size_t n = 0; n < G.N; ++n) {
    OP.hh[n] = hhat_at(n);
    load8(Qe, n, c);
    con2pri(p, c);
    OP.pe[n] = p[4];
    OP.vscale[n] = Vbase_slope(p[4], ucon[n]);
  }
  shock_detector(OP.eta, Qe);
  const double dx = G.dx, dy = G.dy;
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      double h00 = OP.hh[ID(i, j)], hp0 = OP.hh[ID(i + 1, j)], hm0 = OP.hh[ID(i - 1, j)];
      double h0p = OP.hh[ID(i, j + 1)], h0m = OP.hh[ID(i, j - 1)];
      OP.tdiag[ID(i, j)] = h * h * ((0.5 * (hp0 + h00) + 0.5 * (hm0 + h00)) / (dx * dx) +
                                    (0.5 * (h0p + h00) + 0.5 * (h0m + h00)) / (dy * dy));
    }
}

/* Pressure_NestedNewton, implicit_operators.cpp:625-738 */
static void nested_newton(double* p, const double* b) {
  const int dim = (int)G.N;
  const double a = 1.0 / (PP.gamma_plasma - 1.0);
  if (!PP.floor_on && PP.eos_type == IDEAL_GAS) {
    OP.jac = 0;
    gmres(p, b, pressure_ax, pressure_pc, dim);
    return;
  }
  if (PP.floor_on) {
    double bmin = INFINITY;
    for (int n = 0; n < dim; ++n)
      if (b[n] < bmin) bmin = b[n];
    double Vpe;
    if (PP.eos_type == IDEAL_GAS) Vpe = PP.p_floor / (PP.gamma_plasma - 1.0);
    else {
      Vpe = PP.p_floor / (PP.gamma_plasma - 1.0);
      for (int i = 0; i < G.nx; i++)
        for (int j = 0; j < G.ny; j++) {
          double v = Vbase(PP.p_floor, OP.ucon[ID(i, j)]);
          if (isfinite(v) && v > Vpe) Vpe = v;
        }
    }
    double q = Vpe - bmin;
    double M_cor = ((0.0 < q) ? q : 0.0) / ((1.0 - PP.theta) * PP.p_floor);
    double M_base = PP.Mbig_fac / (PP.gamma_plasma - 1.0);
    G.Mbig = (M_base < M_cor) ? M_cor : M_base; /* std::max(M_base, M_cor) */
  }
  double *pf = alloc(dim), *g = alloc(dim), *dp = alloc(dim), *ng = alloc(dim), *Lp = alloc(dim);
  memcpy(pf, p, dim * sizeof(double));
  OP.pfreeze = pf;
  int it;
  double res0 = -1.0;
  for (it = 0; it < PP.Pnewton_max; it++) {
    OP.jac = 0;
    pressure_ax(pf, Lp);
    for (int i = 0; i < G.nx; i++)
      for (int j = 0; j < G.ny; j++) {
        size_t n = ID(i, j);
        g[n] = Lp[n] - a * pf[n] + V_mod(pf[n], OP.ucon[n]) - b[n];
      }
    double res = sqrt(dotv(g, g, dim));
    if (it == 0) res0 = res;
    if (res < PP.Pnewton_tol * res0 + PP.Pnewton_tol) break;
    for (int n = 0; n < dim; ++n) {
      ng[n] = -g[n];
      dp[n] = 0.0;
    }
    OP.jac = 1;
    gmres(dp, ng, pressure_ax, pressure_pc, dim);
    for (int n = 0; n < dim; ++n) pf[n] = pf[n] + dp[n];
  }
  OP.jac = 0;
  memcpy(p, pf, dim * sizeof(double));
  if (PP.floor_on) {
    int nf = 0;
    double pmin = 1e300;
    for (int n = 0; n < dim; ++n) {
      if (p[n] < PP.p_floor) ++nf;
      if (p[n] < pmin) pmin = p[n];
    }
    if (nf > G.max_floored) G.max_floored = nf;
    if (pmin < G.min_p_ever) G.min_p_ever = pmin;
  }
  OP.pfreeze = NULL;
  free(pf); free(g); free(dp); free(ng); free(Lp);
}

/* ------------------------------------------------------------------ */
/* pressure sub-system, imex_subsystems.cpp:76-413                    */
/* ------------------------------------------------------------------ */
static void pressure_rhs(double* b, const double* ucon, const double* rvx, const double* rvy,
                         const double* kin_x, const double* kin_y, const double* kin_z, double h) {
  const double dx = G.dx, dy = G.dy;
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      size_t c = ID(i, j), e = ID(i + 1, j), w = ID(i - 1, j), n = ID(i, j + 1), s = ID(i, j - 1);
      double u5 = ucon[5 * G.N + c], u6 = ucon[6 * G.N + c], u7 = ucon[7 * G.N + c];
      double B2 = u5 * u5 + u6 * u6 + u7 * u7;
      double h00 = OP.hh[c], hp0 = OP.hh[e], hm0 = OP.hh[w], h0p = OP.hh[n], h0m = OP.hh[s];
      double p_star = ucon[4 * G.N + c] - 0.5 * B2;
      b[c] = p_star - 0.5 * (kin_x[c] * kin_x[c] + kin_y[c] * kin_y[c] + kin_z[c] * kin_z[c]) / ucon[c] -
             h * (1 / dx * (0.5 * (hp0 + h00) * 0.5 * (rvx[e] + rvx[c]) - 0.5 * (hm0 + h00) * 0.5 * (rvx[w] + rvx[c])) +
                  (1 / dy * (0.5 * (h0p + h00) * 0.5 * (rvy[n] + rvy[c]) - 0.5 * (h0m + h00) * 0.5 * (rvy[s] + rvy[c]))));
    }
}

static void pre_subsystem_pressure(double* ucon, const double* Qs, const double* Qe, double h, int rks) {
  const size_t N = G.N;
  double *rvx = alloc(N), *rvy = alloc(N), *rvz = alloc(N), *b = alloc(N), *p = alloc(N);
  memcpy(rvx, PL(ucon, 1), N * sizeof(double));
  memcpy(rvy, PL(ucon, 2), N * sizeof(double));
  memcpy(rvz, PL(ucon, 3), N * sizeof(double));
  pressure_setup(ucon, Qe, Qs, h);
  pressure_rhs(b, ucon, rvx, rvy, rvx, rvy, rvz, h);
  memcpy(p, OP.pe, N * sizeof(double));
  nested_newton(p, b);
  const double dx = G.dx, dy = G.dy;
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      size_t c = ID(i, j);
      double flux_xm = 0.5 * (p[ID(i - 1, j)] + p[c]);
      double flux_xp = 0.5 * (p[c] + p[ID(i + 1, j)]);
      ucon[1 * N + c] = rvx[c] - h / dx * (flux_xp - flux_xm);
      double flux_ym = 0.5 * (p[ID(i, j - 1)] + p[c]);
      double flux_yp = 0.5 * (p[c] + p[ID(i, j + 1)]);
      ucon[2 * N + c] = rvy[c] - h / dy * (flux_yp - flux_ym);
    }
  if (PP.PressureSolver == all_correction || (PP.PressureSolver == once_correction && rks == G.R - 1)) {
    pressure_rhs(b, ucon, rvx, rvy, PL(ucon, 1), PL(ucon, 2), PL(ucon, 3), h);
    nested_newton(p, b);
  }
  if (PP.U_update == DefinitionofU) {
    for (size_t c = 0; c < N; ++c) {
      double r = ucon[c], m1 = ucon[N + c], m2 = ucon[2 * N + c], m3 = ucon[3 * N + c];
      double b5 = ucon[5 * N + c], b6 = ucon[6 * N + c], b7 = ucon[7 * N + c];
      ucon[4 * N + c] = Vbase(p[c], r) + 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / r + 0.5 * (b5 * b5 + b6 * b6 + b7 * b7);
    }
  } else {
    /* ConservationofU, imex_subsystems.cpp:303-392: E -= h div(h_e rho v), h_e = e(rho, p) + p / rho
       of the final pressure (ghosts as bound_cond_array) and the corrected momentum */
    for (int i = 0; i < G.nx; i++)
      for (int j = 0; j < G.ny; j++) {
        size_t c = ID(i, j), e = ID(i + 1, j), w = ID(i - 1, j), n = ID(i, j + 1), s = ID(i, j - 1);
        double h_00 = eos_e(ucon[c], p[c]) + p[c] / ucon[c];
        double h_p0 = eos_e(ucon[e], p[e]) + p[e] / ucon[e];
        double h_m0 = eos_e(ucon[w], p[w]) + p[w] / ucon[w];
        double h_0p = eos_e(ucon[n], p[n]) + p[n] / ucon[n];
        double h_0m = eos_e(ucon[s], p[s]) + p[s] / ucon[s];
        double flux_xm = 0.5 * (h_m0 * ucon[N + w] + h_00 * ucon[N + c]);
        double flux_xp = 0.5 * (h_00 * ucon[N + c] + h_p0 * ucon[N + e]);
        double flux_ym = 0.5 * (h_0m * ucon[2 * N + s] + h_00 * ucon[2 * N + c]);
        double flux_yp = 0.5 * (h_00 * ucon[2 * N + c] + h_0p * ucon[2 * N + n]);
        ucon[4 * N + c] = ucon[4 * N + c] - h / (dx) * (flux_xp - flux_xm) - h / (dy) * (flux_yp - flux_ym);
      }
  }
  free(rvx); free(rvy); free(rvz); free(b); free(p);
}

/* ------------------------------------------------------------------ */
/* energy sub-system, PreSubsystem_Energy imex_subsystems.cpp:415-534 */
/* with Energy_Subsystem_AX implicit_operators.cpp:741-795 (periodic) */
/* ------------------------------------------------------------------ */
/* total enthalpy (E + p) / rho, caltotalenthalpy timestep.cpp:232-237 */
static double caltotalenthalpy(const double* c) {
  double pri[8];
  con2pri(pri, c);
  return (c[4] + pri[4]) / pri[0];
}
static void energy_ax(const double* x, double* Ax) {
  const double h = OP.h, dx = G.dx, dy = G.dy, g = PP.gamma_plasma;
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      size_t c = ID(i, j), e = ID(i + 1, j), w = ID(i - 1, j), n = ID(i, j + 1), s = ID(i, j - 1);
      double h00 = OP.hh[c], hp0 = OP.hh[e], hm0 = OP.hh[w], h0p = OP.hh[n], h0m = OP.hh[s];
      double hhp_x = 0.5 * (h00 + hp0), hhm_x = 0.5 * (h00 + hm0);
      double hhp_y = 0.5 * (h00 + h0p), hhm_y = 0.5 * (h00 + h0m);
      double Ei = x[c];
      double r = Ei - (g - 1) * h * h *
                          (1.0 / (dx * dx) * (hhp_x * (x[e] - Ei) - hhm_x * (Ei - x[w])) +
                           1.0 / (dy * dy) * (hhp_y * (x[n] - Ei) - hhm_y * (Ei - x[s])));
      Ax[c] = r * dx * dy;
    }
}
/* precE, imex_subsystems.cpp:487-505: in / (diag dx dy) */
static void energy_pc(const double* in, double* out) {
  for (size_t n = 0; n < G.N; ++n) out[n] = in[n] / OP.tdiag[n];
}
/* the cell enthalpy ratio h(Qe) rho_e / rho of the operator and the Jacobi scale diag dx dy */
static void energy_setup(const double* ucon, const double* Qe, double h) {
  const size_t N = G.N;
  const double dx = G.dx, dy = G.dy, g = PP.gamma_plasma;
  OP.ucon = ucon;
  OP.Qe = Qe;
  OP.h = h;
  free(OP.hh); free(OP.tdiag);
  OP.hh = alloc(N);
  OP.tdiag = alloc(N);
  double c[8];
  for (size_t n = 0; n < N; ++n) {
    load8(Qe, n, c);
    OP.hh[n] = caltotalenthalpy(c) * c[0] / ucon[n];
  }
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      size_t o = ID(i, j);
      double h00 = OP.hh[o], hp0 = OP.hh[ID(i + 1, j)], hm0 = OP.hh[ID(i - 1, j)];
      double h0p = OP.hh[ID(i, j + 1)], h0m = OP.hh[ID(i, j - 1)];
      double hhp_x = 0.5 * (h00 + hp0), hhm_x = 0.5 * (h00 + hm0);
      double hhp_y = 0.5 * (h00 + h0p), hhm_y = 0.5 * (h00 + h0m);
      double diag = 1.0 + (g - 1.0) * h * h * ((hhp_x + hhm_x) / (dx * dx) + (hhp_y + hhm_y) / (dy * dy));
      OP.tdiag[o] = diag * dx * dy;
    }
}
static void pre_subsystem_energy(double* ucon, const double* Qe, double h) {
  const size_t N = G.N;
  const double dx = G.dx, dy = G.dy, g = PP.gamma_plasma;
  energy_setup(ucon, Qe, h);
  double *b = alloc(N), *E = alloc(N);
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      size_t o = ID(i, j), e = ID(i + 1, j), w = ID(i - 1, j), n = ID(i, j + 1), s = ID(i, j - 1);
      double hp0 = OP.hh[e], hm0 = OP.hh[w], h0p = OP.hh[n], h0m = OP.hh[s];
      double U_star = ucon[4 * N + o] - 0.5 * h / dx * (hp0 * ucon[N + e] - hm0 * ucon[N + w]) -
                      0.5 * h / dy * (h0p * ucon[2 * N + n] - h0m * ucon[2 * N + s]);
      b[o] = U_star * dx * dy;
      E[o] = ucon[4 * N + o];
    }
  gmres(E, b, energy_ax, energy_pc, (int)N);
  memcpy(PL(ucon, 4), E, N * sizeof(double));
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      size_t o = ID(i, j);
      ucon[N + o] -= h * (1 / (2 * dx)) * (g - 1) * (E[ID(i + 1, j)] - E[ID(i - 1, j)]);
      ucon[2 * N + o] -= h * (1 / (2 * dy)) * (g - 1) * (E[ID(i, j + 1)] - E[ID(i, j - 1)]);
    }
  free(b); free(E);
}

/* ------------------------------------------------------------------ */
/* magnetic sub-system, B form: imex_subsystems.cpp:537-628,          */
/* Magnetic_Subsystem_AX implicit_operators.cpp:141-353 (GLF)         */
/* ------------------------------------------------------------------ */
#define QE(k, i, j) AT(OP.Qe, k, i, j)
#define UC(k, i, j) AT(OP.ucon, k, i, j)
#define XB(k, i, j) x[(size_t)((k)-5) * G.N + ID(i, j)]

static void magnetic_ax(const double* x, double* Ax) {
  const double h = OP.h, dx = G.dx, dy = G.dy;
  const size_t N = G.N;
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      double rho_p0 = 0.5 * (UC(0, i, j) + UC(0, i + 1, j));
      double rho_m0 = 0.5 * (UC(0, i, j) + UC(0, i - 1, j));
      double rho_0p = 0.5 * (UC(0, i, j) + UC(0, i, j + 1));
      double rho_0m = 0.5 * (UC(0, i, j) + UC(0, i, j - 1));
      double Bxn_p0 = 0.5 * (QE(5, i, j) + QE(5, i + 1, j));
      double Bxn_m0 = 0.5 * (QE(5, i, j) + QE(5, i - 1, j));
      double Bxn_0p = 0.5 * (QE(5, i, j) + QE(5, i, j + 1));
      double Bxn_0m = 0.5 * (QE(5, i, j) + QE(5, i, j - 1));
      double Bxn_pp = 0.25 * (QE(5, i, j) + QE(5, i + 1, j) + QE(5, i, j + 1) + QE(5, i + 1, j + 1));
      double Bxn_pm = 0.25 * (QE(5, i, j) + QE(5, i + 1, j) + QE(5, i, j - 1) + QE(5, i + 1, j - 1));
      double Bxn_mp = 0.25 * (QE(5, i, j) + QE(5, i - 1, j) + QE(5, i, j + 1) + QE(5, i - 1, j + 1));
      double Bxn_mm = 0.25 * (QE(5, i, j) + QE(5, i - 1, j) + QE(5, i, j - 1) + QE(5, i - 1, j - 1));
      double Byn_p0 = 0.5 * (QE(6, i, j) + QE(6, i + 1, j));
      double Byn_m0 = 0.5 * (QE(6, i, j) + QE(6, i - 1, j));
      double Byn_0p = 0.5 * (QE(6, i, j) + QE(6, i, j + 1));
      double Byn_0m = 0.5 * (QE(6, i, j) + QE(6, i, j - 1));
      double Byn_pp = 0.25 * (QE(6, i, j) + QE(6, i + 1, j) + QE(6, i, j + 1) + QE(6, i + 1, j + 1));
      double Byn_pm = 0.25 * (QE(6, i, j) + QE(6, i + 1, j) + QE(6, i, j - 1) + QE(6, i + 1, j - 1));
      double Byn_mp = 0.25 * (QE(6, i, j) + QE(6, i - 1, j) + QE(6, i, j + 1) + QE(6, i - 1, j + 1));
      double Byn_mm = 0.25 * (QE(6, i, j) + QE(6, i - 1, j) + QE(6, i, j - 1) + QE(6, i - 1, j - 1));
      double Bzn_p0 = 0.5 * (QE(7, i, j) + QE(7, i + 1, j));
      double Bzn_m0 = 0.5 * (QE(7, i, j) + QE(7, i - 1, j));
      double Bzn_0p = 0.5 * (QE(7, i, j) + QE(7, i, j + 1));
      double Bzn_0m = 0.5 * (QE(7, i, j) + QE(7, i, j - 1));
      double Bzn_pp = 0.25 * (QE(7, i, j) + QE(7, i + 1, j) + QE(7, i, j + 1) + QE(7, i + 1, j + 1));
      double Bzn_pm = 0.25 * (QE(7, i, j) + QE(7, i + 1, j) + QE(7, i, j - 1) + QE(7, i + 1, j - 1));
      double Bzn_mp = 0.25 * (QE(7, i, j) + QE(7, i - 1, j) + QE(7, i, j + 1) + QE(7, i - 1, j + 1));
      double Bzn_mm = 0.25 * (QE(7, i, j) + QE(7, i - 1, j) + QE(7, i, j - 1) + QE(7, i - 1, j - 1));
      double Bx_pp = 0.25 * (XB(5, i, j) + XB(5, i + 1, j) + XB(5, i, j + 1) + XB(5, i + 1, j + 1));
      double Bx_pm = 0.25 * (XB(5, i, j) + XB(5, i + 1, j) + XB(5, i, j - 1) + XB(5, i + 1, j - 1));
      double Bx_mp = 0.25 * (XB(5, i, j) + XB(5, i - 1, j) + XB(5, i, j + 1) + XB(5, i - 1, j + 1));
      double Bx_mm = 0.25 * (XB(5, i, j) + XB(5, i - 1, j) + XB(5, i, j - 1) + XB(5, i - 1, j - 1));
      double By_pp = 0.25 * (XB(6, i, j) + XB(6, i + 1, j) + XB(6, i, j + 1) + XB(6, i + 1, j + 1));
      double By_pm = 0.25 * (XB(6, i, j) + XB(6, i + 1, j) + XB(6, i, j - 1) + XB(6, i + 1, j - 1));
      double By_mp = 0.25 * (XB(6, i, j) + XB(6, i - 1, j) + XB(6, i, j + 1) + XB(6, i - 1, j + 1));
      double By_mm = 0.25 * (XB(6, i, j) + XB(6, i - 1, j) + XB(6, i, j - 1) + XB(6, i - 1, j - 1));
      double Bz_pp = 0.25 * (XB(7, i, j) + XB(7, i + 1, j) + XB(7, i, j + 1) + XB(7, i + 1, j + 1));
      double Bz_pm = 0.25 * (XB(7, i, j) + XB(7, i + 1, j) + XB(7, i, j - 1) + XB(7, i + 1, j - 1));
      double Bz_mp = 0.25 * (XB(7, i, j) + XB(7, i - 1, j) + XB(7, i, j + 1) + XB(7, i - 1, j + 1));
      double Bz_mm = 0.25 * (XB(7, i, j) + XB(7, i - 1, j) + XB(7, i, j - 1) + XB(7, i - 1, j - 1));

      /* dot products Qe(cell) . x(cell) at the cell and its 4 neighbours */
#define QX(ii, jj) (0.5 * (QE(5, ii, jj) * XB(5, ii, jj) + QE(6, ii, jj) * XB(6, ii, jj) + QE(7, ii, jj) * XB(7, ii, jj)))
      double Bx_1 = Bxn_0p / rho_0p *
                    (1 / dx * (Bxn_pp * By_pp - Bxn_mp * By_mp) -
                     1 / dy * ((QX(i, j + 1) - QE(6, i, j + 1) * XB(6, i, j + 1)) - (QX(i, j) - QE(6, i, j) * XB(6, i, j))));
      double Bx_2 = Byn_0p / rho_0p *
                    (1 / dx * ((0.5 * (Bxn_pp * Bx_pp + Byn_pp * By_pp + Bzn_pp * Bz_pp) - Bxn_pp * Bx_pp) -
                               (0.5 * (Bxn_mp * Bx_mp + Byn_mp * By_mp + Bzn_mp * Bz_mp) - Bxn_mp * Bx_mp)) -
                     1 / dy * (QE(6, i, j + 1) * XB(5, i, j + 1) - QE(6, i, j) * XB(5, i, j)));
      double Bx_3 = Bxn_0m / rho_0m *
                    (1 / dx * (Bxn_pm * By_pm - Bxn_mm * By_mm) -
                     1 / dy * ((QX(i, j) - QE(6, i, j) * XB(6, i, j)) - (QX(i, j - 1) - QE(6, i, j - 1) * XB(6, i, j - 1))));
      double Bx_4 = Byn_0m / rho_0m *
                    (1 / dx * ((0.5 * (Bxn_pm * Bx_pm + Byn_pm * By_pm + Bzn_pm * Bz_pm) - Bxn_pm * Bx_pm) -
                               (0.5 * (Bxn_mm * Bx_mm + Byn_mm * By_mm + Bzn_mm * Bz_mm) - Bxn_mm * Bx_mm)) -
                     1 / dy * (QE(6, i, j) * XB(5, i, j) - QE(6, i, j - 1) * XB(5, i, j - 1)));
      double ax5 = XB(5, i, j) + (h * h / dy) * ((Bx_1 + Bx_2) - (Bx_3 + Bx_4));

      double By_1 = Byn_p0 / rho_p0 *
                    (-1 / dx * ((QX(i + 1, j) - QE(5, i + 1, j) * XB(5, i + 1, j)) - (QX(i, j) - QE(5, i, j) * XB(5, i, j))) +
                     1 / dy * (Bxn_pp * By_pp - Bxn_pm * By_pm));
      double By_2 = Bxn_p0 / rho_p0 *
                    (-1 / dx * (QE(5, i + 1, j) * XB(6, i + 1, j) - QE(5, i, j) * XB(6, i, j)) +
                     1 / dy * ((0.5 * (Bxn_pp * Bx_pp + Byn_pp * By_pp + Bzn_pp * Bz_pp) - Byn_pp * By_pp) -
                               (0.5 * (Bxn_pm * Bx_pm + Byn_pm * By_pm + Bzn_pm * Bz_pm) - Byn_pm * By_pm)));
      double By_3 = Byn_m0 / rho_m0 *
                    (-1 / dx * ((QX(i, j) - QE(5, i, j) * XB(5, i, j)) - (QX(i - 1, j) - QE(5, i - 1, j) * XB(5, i - 1, j))) +
                     1 / dy * (Bxn_mp * By_mp - Bxn_mm * By_mm));
      double By_4 = Bxn_m0 / rho_m0 *
                    (-1 / dx * (QE(5, i, j) * XB(6, i, j) - QE(5, i - 1, j) * XB(6, i - 1, j)) +
                     1 / dy * ((0.5 * (Bxn_mp * Bx_mp + Byn_mp * By_mp + Bzn_mp * Bz_mp) - Byn_mp * By_mp) -
                               (0.5 * (Bxn_mm * Bx_mm + Byn_mm * By_mm + Bzn_mm * Bz_mm) - Byn_mm * By_mm)));
      double ax6 = XB(6, i, j) + (h * h / dx) * ((By_1 + By_2) - (By_3 + By_4));

      double Bz_1 = Bzn_p0 / rho_p0 *
                    (-1 / dx * ((QX(i + 1, j) - QE(5, i + 1, j) * XB(5, i + 1, j)) - (QX(i, j) - QE(5, i, j) * XB(5, i, j))) +
                     1 / dy * (Byn_pp * Bx_pp - Byn_pm * Bx_pm));
      double Bz_2 = Bxn_p0 / rho_p0 *
                    (-1 / dx * (QE(5, i + 1, j) * XB(7, i + 1, j) - QE(5, i, j) * XB(7, i, j)) -
                     1 / dy * (Byn_pp * Bz_pp - Byn_pm * Bz_pm));
      double Bz_3 = Bzn_m0 / rho_m0 *
                    (-1 / dx * ((QX(i, j) - QE(5, i, j) * XB(5, i, j)) - (QX(i - 1, j) - QE(5, i - 1, j) * XB(5, i - 1, j))) +
                     1 / dy * (Byn_mp * Bx_mp - Byn_mm * Bx_mm));
      double Bz_4 = Bxn_m0 / rho_m0 *
                    (-1 / dx * (QE(5, i, j) * XB(7, i, j) - QE(5, i - 1, j) * XB(7, i - 1, j)) -
                     1 / dy * (Byn_mp * Bz_mp - Byn_mm * Bz_mm));
      double Bz_5 = Bzn_0p / rho_0p *
                    (1 / dx * (Bxn_pp * By_pp - Bxn_mp * By_mp) -
                     1 / dy * ((QX(i, j + 1) - QE(6, i, j + 1) * XB(6, i, j + 1)) - (QX(i, j) - QE(6, i, j) * XB(6, i, j))));
      double Bz_6 = Byn_0p / rho_0p *
                    (-1 / dx * (Bxn_pp * Bz_pp - Bxn_mp * Bz_mp) -
                     1 / dy * (QE(6, i, j + 1) * XB(7, i, j + 1) - QE(6, i, j) * XB(7, i, j)));
      double Bz_7 = Bzn_0m / rho_0m *
                    (1 / dx * (Bxn_pm * By_pm - Bxn_mm * By_mm) -
                     1 / dy * ((QX(i, j) - QE(6, i, j) * XB(6, i, j)) - (QX(i, j - 1) - QE(6, i, j - 1) * XB(6, i, j - 1))));
      double Bz_8 = Byn_0m / rho_0m *
                    (-1 / dx * (Bxn_pm * Bz_pm - Bxn_mm * Bz_mm) -
                     1 / dy * (QE(6, i, j) * XB(7, i, j) - QE(6, i, j - 1) * XB(7, i, j - 1)));
#undef QX
      double ax7 = XB(7, i, j) + h * h / dx * ((Bz_1 + Bz_2) - (Bz_3 + Bz_4)) + h * h / dy * ((Bz_5 + Bz_6) - (Bz_7 + Bz_8));

      double nu_x = G.B_max_x * dx, nu_y = G.B_max_y * dy;
      double nu_x_p = 0, nu_x_m = 0, nu_y_p = 0, nu_y_m = 0;
      if (!PP.GLF) { /* implicit_operators.cpp:323-352 */
        double b_x = lf_speed_at(OP.Qe, i, j, 0), b_y = lf_speed_at(OP.Qe, i, j, 1);
        nu_x_p = fmax(fabs(b_x), fabs(lf_speed_at(OP.Qe, i + 1, j, 0))) * dx;
        nu_x_m = fmax(fabs(b_x), fabs(lf_speed_at(OP.Qe, i - 1, j, 0))) * dx;
        nu_y_p = fmax(fabs(b_y), fabs(lf_speed_at(OP.Qe, i, j + 1, 1))) * dy;
        nu_y_m = fmax(fabs(b_y), fabs(lf_speed_at(OP.Qe, i, j - 1, 1))) * dy;
      }
      for (int k = 5; k <= 7; ++k) {
        double lap;
        if (PP.GLF)
          lap = nu_x / (dx * dx) * (XB(k, i - 1, j) - 2.0 * XB(k, i, j) + XB(k, i + 1, j)) +
                nu_y / (dy * dy) * (XB(k, i, j - 1) - 2.0 * XB(k, i, j) + XB(k, i, j + 1));
        else
          lap = 1 / (dx * dx) * (nu_x_p * (XB(k, i + 1, j) - XB(k, i, j)) - nu_x_m * (XB(k, i, j) - XB(k, i - 1, j))) +
                1 / (dy * dy) * (nu_y_p * (XB(k, i, j + 1) - XB(k, i, j)) - nu_y_m * (XB(k, i, j) - XB(k, i, j - 1)));
        double base = k == 5 ? ax5 : (k == 6 ? ax6 : ax7);
        Ax[(size_t)(k - 5) * N + ID(i, j)] = base - h * lap;
      }
    }
}

/* B* right-hand side, imex_subsystems.cpp:549-615 */
static void magnetic_rhs_B(double* b, const double* ucon, const double* Qe, const double* Qs, const double* pe,
                           double h) {
  const double dx = G.dx, dy = G.dy;
  const size_t N = G.N;
#define U(k, ii, jj) AT(ucon, k, ii, jj)
#define Q(k, ii, jj) AT(Qe, k, ii, jj)
#define PE(ii, jj) pe[ID(ii, jj)]
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      double rho_p0 = 0.5 * (U(0, i, j) + U(0, i + 1, j)), rho_m0 = 0.5 * (U(0, i, j) + U(0, i - 1, j));
      double rho_0p = 0.5 * (U(0, i, j) + U(0, i, j + 1)), rho_0m = 0.5 * (U(0, i, j) + U(0, i, j - 1));
      double rvx_p0 = 0.5 * (U(1, i, j) + U(1, i + 1, j)), rvx_m0 = 0.5 * (U(1, i, j) + U(1, i - 1, j));
      double rvx_0p = 0.5 * (U(1, i, j) + U(1, i, j + 1)), rvx_0m = 0.5 * (U(1, i, j) + U(1, i, j - 1));
      double rvy_p0 = 0.5 * (U(2, i, j) + U(2, i + 1, j)), rvy_m0 = 0.5 * (U(2, i, j) + U(2, i - 1, j));
      double rvy_0p = 0.5 * (U(2, i, j) + U(2, i, j + 1)), rvy_0m = 0.5 * (U(2, i, j) + U(2, i, j - 1));
      double rvz_p0 = 0.5 * (U(3, i, j) + U(3, i + 1, j)), rvz_m0 = 0.5 * (U(3, i, j) + U(3, i - 1, j));
      double rvz_0p = 0.5 * (U(3, i, j) + U(3, i, j + 1)), rvz_0m = 0.5 * (U(3, i, j) + U(3, i, j - 1));
      double p_pp = 0.25 * (PE(i, j) + PE(i + 1, j) + PE(i, j + 1) + PE(i + 1, j + 1));
      double p_pm = 0.25 * (PE(i, j) + PE(i + 1, j) + PE(i, j - 1) + PE(i + 1, j - 1));
      double p_mp = 0.25 * (PE(i, j) + PE(i - 1, j) + PE(i, j + 1) + PE(i - 1, j + 1));
      double p_mm = 0.25 * (PE(i, j) + PE(i - 1, j) + PE(i, j - 1) + PE(i - 1, j - 1));
      double Bxn_p0 = 0.5 * (Q(5, i, j) + Q(5, i + 1, j)), Bxn_m0 = 0.5 * (Q(5, i, j) + Q(5, i - 1, j));
      double Bxn_0p = 0.5 * (Q(5, i, j) + Q(5, i, j + 1)), Bxn_0m = 0.5 * (Q(5, i, j) + Q(5, i, j - 1));
      double Byn_p0 = 0.5 * (Q(6, i, j) + Q(6, i + 1, j)), Byn_m0 = 0.5 * (Q(6, i, j) + Q(6, i - 1, j));
      double Byn_0p = 0.5 * (Q(6, i, j) + Q(6, i, j + 1)), Byn_0m = 0.5 * (Q(6, i, j) + Q(6, i, j - 1));
      double Bzn_p0 = 0.5 * (Q(7, i, j) + Q(7, i + 1, j)), Bzn_m0 = 0.5 * (Q(7, i, j) + Q(7, i - 1, j));
      double Bzn_0p = 0.5 * (Q(7, i, j) + Q(7, i, j + 1)), Bzn_0m = 0.5 * (Q(7, i, j) + Q(7, i, j - 1));
      double Bx_star = AT(Qs, 5, i, j) -
                       (h / dy) * ((Bxn_0p / rho_0p * (rvy_0p - (h / dy) * (PE(i, j + 1) - PE(i, j))) -
                                    Byn_0p / rho_0p * (rvx_0p - h / dx * (p_pp - p_mp))) -
                                   (Bxn_0m / rho_0m * (rvy_0m - (h / dy) * (PE(i, j) - PE(i, j - 1))) -
                                    Byn_0m / rho_0m * (rvx_0m - h / dx * (p_pm - p_mm))));
      double By_star = AT(Qs, 6, i, j) -
                       (h / dx) * ((Byn_p0 / rho_p0 * (rvx_p0 - (h / dx) * (PE(i + 1, j) - PE(i, j))) -
                                    Bxn_p0 / rho_p0 * (rvy_p0 - h / dy * (p_pp - p_pm))) -
                                   (Byn_m0 / rho_m0 * (rvx_m0 - (h / dx) * (PE(i, j) - PE(i - 1, j))) -
                                    Bxn_m0 / rho_m0 * (rvy_m0 - h / dy * (p_mp - p_mm))));
      double Bz1 = ((Bzn_p0 / rho_p0 * (rvx_p0 - h / dx * (PE(i + 1, j) - PE(i, j))) - Bxn_p0 / rho_p0 * (rvz_p0)) -
                    (Bzn_m0 / rho_m0 * (rvx_m0 - h / dx * (PE(i, j) - PE(i - 1, j))) - Bxn_m0 / rho_m0 * (rvz_m0)));
      double Bz2 = ((Bzn_0p / rho_0p * (rvy_0p - h / dy * (PE(i, j + 1) - PE(i, j))) - Byn_0p / rho_0p * (rvz_0p)) -
                    (Bzn_0m / rho_0m * (rvy_0m - h / dy * (PE(i, j) - PE(i, j - 1))) - Byn_0m / rho_0m * (rvz_0m)));
      double Bz_star = AT(Qs, 7, i, j) - (h / dx) * Bz1 - (h / dy) * Bz2;
      size_t c = ID(i, j);
      b[c] = Bx_star;
      b[N + c] = By_star;
      b[2 * N + c] = Bz_star;
    }
#undef U
#undef Q
#undef PE
}

/* CollectMagFluxes, ct_flux.cpp:5-130 (GLF, periodic) */
static void collect_mag_fluxes(double* Fx, double* Fy, const double* ucon, const double* Qe, const double* pe,
                               double h) {
  const double dx = G.dx, dy = G.dy;
#define U(k, ii, jj) AT(ucon, k, ii, jj)
#define Q(k, ii, jj) AT(Qe, k, ii, jj)
#define PE(ii, jj) pe[ID(ii, jj)]
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      double rho_p0 = 0.5 * (U(0, i, j) + U(0, i + 1, j)), rho_0p = 0.5 * (U(0, i, j) + U(0, i, j + 1));
      double rvx_p0 = 0.5 * (U(1, i, j) + U(1, i + 1, j)), rvy_p0 = 0.5 * (U(2, i, j) + U(2, i + 1, j));
      double rvx_0p = 0.5 * (U(1, i, j) + U(1, i, j + 1)), rvy_0p = 0.5 * (U(2, i, j) + U(2, i, j + 1));
      double p_pp = 0.25 * (PE(i, j) + PE(i + 1, j) + PE(i, j + 1) + PE(i + 1, j + 1));
      double p_pm = 0.25 * (PE(i, j) + PE(i + 1, j) + PE(i, j - 1) + PE(i + 1, j - 1));
      double p_mp = 0.25 * (PE(i, j) + PE(i - 1, j) + PE(i, j + 1) + PE(i - 1, j + 1));
      double Bxn_p0 = 0.5 * (Q(5, i, j) + Q(5, i + 1, j)), Byn_p0 = 0.5 * (Q(6, i, j) + Q(6, i + 1, j));
      double Bxn_0p = 0.5 * (Q(5, i, j) + Q(5, i, j + 1)), Byn_0p = 0.5 * (Q(6, i, j) + Q(6, i, j + 1));
      double Bxn_pp = 0.25 * (Q(5, i, j) + Q(5, i + 1, j) + Q(5, i, j + 1) + Q(5, i + 1, j + 1));
      double Bxn_pm = 0.25 * (Q(5, i, j) + Q(5, i + 1, j) + Q(5, i, j - 1) + Q(5, i + 1, j - 1));
      double Bxn_mp = 0.25 * (Q(5, i, j) + Q(5, i - 1, j) + Q(5, i, j + 1) + Q(5, i - 1, j + 1));
      double Byn_pp = 0.25 * (Q(6, i, j) + Q(6, i + 1, j) + Q(6, i, j + 1) + Q(6, i + 1, j + 1));
      double Byn_pm = 0.25 * (Q(6, i, j) + Q(6, i + 1, j) + Q(6, i, j - 1) + Q(6, i + 1, j - 1));
      double Byn_mp = 0.25 * (Q(6, i, j) + Q(6, i - 1, j) + Q(6, i, j + 1) + Q(6, i - 1, j + 1));
      double Bzn_pp = 0.25 * (Q(7, i, j) + Q(7, i + 1, j) + Q(7, i, j + 1) + Q(7, i + 1, j + 1));
      double Bzn_pm = 0.25 * (Q(7, i, j) + Q(7, i + 1, j) + Q(7, i, j - 1) + Q(7, i + 1, j - 1));
      double Bzn_mp = 0.25 * (Q(7, i, j) + Q(7, i - 1, j) + Q(7, i, j + 1) + Q(7, i - 1, j + 1));
      double Bx1_pp = 0.25 * (U(5, i, j) + U(5, i + 1, j) + U(5, i, j + 1) + U(5, i + 1, j + 1));
      double Bx1_pm = 0.25 * (U(5, i, j) + U(5, i + 1, j) + U(5, i, j - 1) + U(5, i + 1, j - 1));
      double Bx1_mp = 0.25 * (U(5, i, j) + U(5, i - 1, j) + U(5, i, j + 1) + U(5, i - 1, j + 1));
      double By1_pp = 0.25 * (U(6, i, j) + U(6, i + 1, j) + U(6, i, j + 1) + U(6, i + 1, j + 1));
      double By1_pm = 0.25 * (U(6, i, j) + U(6, i + 1, j) + U(6, i, j - 1) + U(6, i + 1, j - 1));
      double By1_mp = 0.25 * (U(6, i, j) + U(6, i - 1, j) + U(6, i, j + 1) + U(6, i - 1, j + 1));
      double Bz1_pp = 0.25 * (U(7, i, j) + U(7, i + 1, j) + U(7, i, j + 1) + U(7, i + 1, j + 1));
      double Bz1_pm = 0.25 * (U(7, i, j) + U(7, i + 1, j) + U(7, i, j - 1) + U(7, i + 1, j - 1));
      double Bz1_mp = 0.25 * (U(7, i, j) + U(7, i - 1, j) + U(7, i, j + 1) + U(7, i - 1, j + 1));
#define QU(ii, jj) (0.5 * (Q(5, ii, jj) * U(5, ii, jj) + Q(6, ii, jj) * U(6, ii, jj) + Q(7, ii, jj) * U(7, ii, jj)))
      double Fn_x = Byn_p0 / rho_p0 * (rvx_p0 - (h / dx) * (PE(i + 1, j) - PE(i, j))) -
                    Bxn_p0 / rho_p0 * (rvy_p0 - (h / dy) * (p_pp - p_pm));
      double By_1 = Byn_p0 / rho_p0 *
                    (-1.0 / dx * ((QU(i + 1, j) - Q(5, i + 1, j) * U(5, i + 1, j)) - (QU(i, j) - Q(5, i, j) * U(5, i, j))) +
                     1.0 / dy * (Bxn_pp * By1_pp - Bxn_pm * By1_pm));
      double By_2 = Bxn_p0 / rho_p0 *
                    (-1.0 / dx * (Q(5, i + 1, j) * U(6, i + 1, j) - Q(5, i, j) * U(6, i, j)) +
                     1.0 / dy * ((0.5 * (Bxn_pp * Bx1_pp + Byn_pp * By1_pp + Bzn_pp * Bz1_pp) - Byn_pp * By1_pp) -
                                 (0.5 * (Bxn_pm * Bx1_pm + Byn_pm * By1_pm + Bzn_pm * Bz1_pm) - Byn_pm * By1_pm)));
      double nu_x = G.B_max_x * dx;
      if (!PP.GLF) nu_x = fmax(fabs(lf_speed_at(Qe, i, j, 0)), fabs(lf_speed_at(Qe, i + 1, j, 0))) * dx;
      double Fdiff_x = -nu_x * (U(6, i + 1, j) - U(6, i, j)) / dx;
      Fx[ID(i, j)] = Fn_x + h * (By_1 + By_2) + Fdiff_x;
      double Fn_y = Bxn_0p / rho_0p * (rvy_0p - (h / dy) * (PE(i, j + 1) - PE(i, j))) -
                    Byn_0p / rho_0p * (rvx_0p - (h / dx) * (p_pp - p_mp));
      double Bx_1 = Bxn_0p / rho_0p *
                    (1.0 / dx * (Bxn_pp * By1_pp - Bxn_mp * By1_mp) -
                     1.0 / dy * ((QU(i, j + 1) - Q(6, i, j + 1) * U(6, i, j + 1)) - (QU(i, j) - Q(6, i, j) * U(6, i, j))));
      double Bx_2 = Byn_0p / rho_0p *
                    (1.0 / dx * ((0.5 * (Bxn_pp * Bx1_pp + Byn_pp * By1_pp + Bzn_pp * Bz1_pp) - Bxn_pp * Bx1_pp) -
                                 (0.5 * (Bxn_mp * Bx1_mp + Byn_mp * By1_mp + Bzn_mp * Bz1_mp) - Bxn_mp * Bx1_mp)) -
                     1.0 / dy * (Q(6, i, j + 1) * U(5, i, j + 1) - Q(6, i, j) * U(5, i, j)));
#undef QU
      double nu_y = G.B_max_y * dy;
      if (!PP.GLF) nu_y = fmax(fabs(lf_speed_at(Qe, i, j, 1)), fabs(lf_speed_at(Qe, i, j + 1, 1))) * dy;
      double Fdiff_y = -nu_y * (U(5, i, j + 1) - U(5, i, j)) / dy;
      Fy[ID(i, j)] = Fn_y + h * (Bx_1 + Bx_2) + Fdiff_y;
    }
#undef U
#undef Q
#undef PE
}

static void mag_subsystem_B(double* ucon, const double* Qs, const double* Qe, double h, double* Fx, double* Fy) {
  const size_t N = G.N;
  double *pri = alloc(8 * N), *b = alloc(3 * N), *x = alloc(3 * N), *pe = alloc(N);
  grid_con2pri(pri, Qe);
  memcpy(pe, PL(pri, 4), N * sizeof(double));
  magnetic_rhs_B(b, ucon, Qe, Qs, pe, h);
  memcpy(x, PL(Qe, 5), 3 * N * sizeof(double));
  OP.ucon = ucon;
  OP.Qe = Qe;
  OP.Qs = Qs;
  OP.h = h;
  gmres(x, b, magnetic_ax, NULL, (int)(3 * N));
  memcpy(PL(ucon, 5), x, 3 * N * sizeof(double));
  collect_mag_fluxes(Fx, Fy, ucon, Qe, pe, h);
  free(pri); free(b); free(x); free(pe);
}

/* ------------------------------------------------------------------ */
/* magnetic sub-system, A form: imex_subsystems.cpp:5-74,             */
/* Magnetic_Subsystem_potential_AX implicit_operators.cpp:355-503     */
/* ------------------------------------------------------------------ */
static void potential_ax(const double* x, double* Ax) {
  const double h = OP.h, dx = G.dx, dy = G.dy;
  const size_t N = G.N;
#define AG(ii, jj, k) agh(x + (size_t)(k)*N, ii, jj)
#define Q(k, ii, jj) AT(OP.Qe, k, ii, jj)
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      double Bxn_00 = Q(5, i, j), Byn_00 = Q(6, i, j), Bzn_00 = Q(7, i, j);
      double Bxn_P0 = Q(5, i + 1, j), Byn_P0 = Q(6, i + 1, j), Bzn_P0 = Q(7, i + 1, j);
      double Bxn_M0 = Q(5, i - 1, j), Byn_M0 = Q(6, i - 1, j), Bzn_M0 = Q(7, i - 1, j);
      double Bxn_0P = Q(5, i, j + 1), Byn_0P = Q(6, i, j + 1), Bzn_0P = Q(7, i, j + 1);
      double Bxn_0M = Q(5, i, j - 1), Byn_0M = Q(6, i, j - 1), Bzn_0M = Q(7, i, j - 1);
      double rho_00 = AT(OP.ucon, 0, i, j);
      double bx_P0 = (AG(i + 1, j + 1, 2) - AG(i + 1, j - 1, 2)) / (2.0 * dy);
      double by_P0 = -(AG(i + 2, j, 2) - AG(i, j, 2)) / (2.0 * dx);
      double bz_P0 = (AG(i + 2, j, 1) - AG(i, j, 1)) / (2.0 * dx) - (AG(i + 1, j + 1, 0) - AG(i + 1, j - 1, 0)) / (2.0 * dy);
      double bx_M0 = (AG(i - 1, j + 1, 2) - AG(i - 1, j - 1, 2)) / (2.0 * dy);
      double by_M0 = -(AG(i, j, 2) - AG(i - 2, j, 2)) / (2.0 * dx);
      double bz_M0 = (AG(i, j, 1) - AG(i - 2, j, 1)) / (2.0 * dx) - (AG(i - 1, j + 1, 0) - AG(i - 1, j - 1, 0)) / (2.0 * dy);
      double bx_0P = (AG(i, j + 2, 2) - AG(i, j, 2)) / (2.0 * dy);
      double by_0P = -(AG(i + 1, j + 1, 2) - AG(i - 1, j + 1, 2)) / (2.0 * dx);
      double bz_0P = (AG(i + 1, j + 1, 1) - AG(i - 1, j + 1, 1)) / (2.0 * dx) - (AG(i, j + 2, 0) - AG(i, j, 0)) / (2.0 * dy);
      double bx_0M = (AG(i, j, 2) - AG(i, j - 2, 2)) / (2.0 * dy);
      double by_0M = -(AG(i + 1, j - 1, 2) - AG(i - 1, j - 1, 2)) / (2.0 * dx);
      double bz_0M = (AG(i + 1, j - 1, 1) - AG(i - 1, j - 1, 1)) / (2.0 * dx) - (AG(i, j, 0) - AG(i, j - 2, 0)) / (2.0 * dy);
      double bdot_P0 = Bxn_P0 * bx_P0 + Byn_P0 * by_P0 + Bzn_P0 * bz_P0;
      double Txx_P0 = bdot_P0 / 2.0 - Bxn_P0 * bx_P0, Tyx_P0 = -Bxn_P0 * by_P0, Tzx_P0 = -Bxn_P0 * bz_P0;
      double bdot_M0 = Bxn_M0 * bx_M0 + Byn_M0 * by_M0 + Bzn_M0 * bz_M0;
      double Txx_M0 = bdot_M0 / 2.0 - Bxn_M0 * bx_M0, Tyx_M0 = -Bxn_M0 * by_M0, Tzx_M0 = -Bxn_M0 * bz_M0;
      double bdot_0P = Bxn_0P * bx_0P + Byn_0P * by_0P + Bzn_0P * bz_0P;
      double Txy_0P = -Byn_0P * bx_0P, Tyy_0P = bdot_0P / 2.0 - Byn_0P * by_0P, Tzy_0P = -Byn_0P * bz_0P;
      double bdot_0M = Bxn_0M * bx_0M + Byn_0M * by_0M + Bzn_0M * bz_0M;
      double Txy_0M = -Byn_0M * bx_0M, Tyy_0M = bdot_0M / 2.0 - Byn_0M * by_0M, Tzy_0M = -Byn_0M * bz_0M;
      double divT_x = (Txx_P0 - Txx_M0) / (2.0 * dx) + (Txy_0P - Txy_0M) / (2.0 * dy);
      double divT_y = (Tyx_P0 - Tyx_M0) / (2.0 * dx) + (Tyy_0P - Tyy_0M) / (2.0 * dy);
      double divT_z = (Tzx_P0 - Tzx_M0) / (2.0 * dx) + (Tzy_0P - Tzy_0M) / (2.0 * dy);
      double Fx = h / rho_00 * divT_x, Fy = h / rho_00 * divT_y, Fz = h / rho_00 * divT_z;
      double cross_x = Byn_00 * Fz - Bzn_00 * Fy;
      double cross_y = Bzn_00 * Fx - Bxn_00 * Fz;
      double cross_z = Bxn_00 * Fy - Byn_00 * Fx;
      double lap[3] = {0.0, 0.0, 0.0};
      if (PP.GLF) {
        double nu_x = OP.gmax_bx * dx, nu_y = OP.gmax_by * dy;
        for (int k = 0; k < 3; ++k)
          lap[k] = nu_x / (dx * dx) * (AG(i - 1, j, k) - 2.0 * AG(i, j, k) + AG(i + 1, j, k)) +
                   nu_y / (dy * dy) * (AG(i, j - 1, k) - 2.0 * AG(i, j, k) + AG(i, j + 1, k));
      } else { /* face averages of the speeds of prim(Qs), implicit_operators.cpp:472-490 */
        double b_x = lf_speed_at(OP.Qs, i, j, 0), b_y = lf_speed_at(OP.Qs, i, j, 1);
        double nu_xp = 0.5 * (fabs(b_x) + fabs(lf_speed_at(OP.Qs, i + 1, j, 0))) * dx;
        double nu_xm = 0.5 * (fabs(b_x) + fabs(lf_speed_at(OP.Qs, i - 1, j, 0))) * dx;
        double nu_yp = 0.5 * (fabs(b_y) + fabs(lf_speed_at(OP.Qs, i, j + 1, 1))) * dy;
        double nu_ym = 0.5 * (fabs(b_y) + fabs(lf_speed_at(OP.Qs, i, j - 1, 1))) * dy;
        for (int k = 0; k < 3; ++k)
          lap[k] = 1.0 / (dx * dx) * (nu_xp * (AG(i + 1, j, k) - AG(i, j, k)) - nu_xm * (AG(i, j, k) - AG(i - 1, j, k))) +
                   1.0 / (dy * dy) * (nu_yp * (AG(i, j + 1, k) - AG(i, j, k)) - nu_ym * (AG(i, j, k) - AG(i, j - 1, k)));
      }
      if (!PP.add_bvisc) lap[0] = lap[1] = lap[2] = 0.0;
      size_t c = ID(i, j);
      Ax[c] = AG(i, j, 0) - h * cross_x - h * lap[0];
      Ax[N + c] = AG(i, j, 1) - h * cross_y - h * lap[1];
      Ax[2 * N + c] = AG(i, j, 2) - h * cross_z - h * lap[2];
    }
#undef AG
#undef Q
}

/* global A-viscosity maxima from prim(Qs) over real cells, implicit_operators.cpp:364-374 */
static void potential_gmax(const double* Qs) {
  double c[8], p[8];
  OP.gmax_bx = 0.0;
  OP.gmax_by = 0.0;
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      load8(Qs, ID(i, j), c);
      con2pri(p, c);
      double Bsq = p[5] * p[5] + p[6] * p[6] + p[7] * p[7];
      double bxv = 0.5 * (fabs(p[1]) + sqrt(p[1] * p[1] + 4.0 * Bsq / p[0]));
      double byv = 0.5 * (fabs(p[2]) + sqrt(p[2] * p[2] + 4.0 * Bsq / p[0]));
      if (bxv > OP.gmax_bx) OP.gmax_bx = bxv;
      if (byv > OP.gmax_by) OP.gmax_by = byv;
    }
}

static void mag_subsystem_A(double* ucon, const double* Qs, const double* Qe, double* A, const double* A_s, double h) {
  const size_t N = G.N;
  const double dx = G.dx, dy = G.dy;
  double *pri = alloc(8 * N), *b = alloc(3 * N), *x = alloc(3 * N);
  grid_con2pri(pri, Qe);
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      size_t c = ID(i, j);
      double Bxn = Qe[5 * N + c], Byn = Qe[6 * N + c], Bzn = Qe[7 * N + c];
      double rho = ucon[c];
      double Sx = ucon[N + c] / rho - h / rho * (AT(pri, 4, i + 1, j) - AT(pri, 4, i - 1, j)) / (2.0 * dx);
      double Sy = ucon[2 * N + c] / rho - h / rho * (AT(pri, 4, i, j + 1) - AT(pri, 4, i, j - 1)) / (2.0 * dy);
      double Sz = ucon[3 * N + c] / rho;
      b[c] = A_s[c] - h * (Byn * Sz - Bzn * Sy);
      b[N + c] = A_s[N + c] - h * (Bzn * Sx - Bxn * Sz);
      b[2 * N + c] = A_s[2 * N + c] - h * (Bxn * Sy - Byn * Sx);
    }
  memcpy(x, A, 3 * N * sizeof(double));
  OP.ucon = ucon;
  OP.Qe = Qe;
  OP.Qs = Qs;
  OP.h = h;
  potential_gmax(Qs);
  gmres(x, b, potential_ax, NULL, (int)(3 * N));
  memcpy(A, x, 3 * N * sizeof(double));
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      size_t c = ID(i, j);
      const double *A0 = A, *A1 = A + N, *A2 = A + 2 * N;
      ucon[5 * N + c] = 1 / (2.0 * dy) * (agh(A2, i, j + 1) - agh(A2, i, j - 1));
      ucon[6 * N + c] = -1 / (2.0 * dx) * (agh(A2, i + 1, j) - agh(A2, i - 1, j));
      ucon[7 * N + c] = 1 / (2.0 * dx) * (agh(A1, i + 1, j) - agh(A1, i - 1, j)) -
                        1 / (2.0 * dy) * (agh(A0, i, j + 1) - agh(A0, i, j - 1));
    }
  free(pri); free(b); free(x);
}

/* ------------------------------------------------------------------ */
/* constrained transport                                              */
/* ------------------------------------------------------------------ */
/* CT_CornerAssemble, constrained_transport.cpp:147-164: the corner (i+1/2, j+1/2) for
 * i, j >= -1.  Ez_bar holds its ghost corners by bound_cond_array (a clamp or a wrap of the
 * corner index), the correction terms read the edge and cell EMFs at the corner itself. */
static double corner_at(int i, int j, const double* Ep0, const double* E0p, const double* Et) {
  const double dx = G.dx, dy = G.dy;
  const int bi = i < 0 ? (G.xclamp ? 0 : G.nx + i) : i, bj = j < 0 ? (G.yclamp ? 0 : G.ny + j) : j;
#define E(a, ii, jj) a[ID(ii, jj)]
  double bar = 0.25 * (E(Ep0, bi, bj) + E(Ep0, bi, bj + 1) + E(E0p, bi, bj) + E(E0p, bi + 1, bj));
  double t1 = 0.5 * ((E(Ep0, i, j) - E(Et, i, j)) / (dx / 2.0) + (E(Ep0, i, j + 1) - E(Et, i, j + 1)) / (dx / 2.0));
  double t2 = 0.5 * ((E(Et, i + 1, j) - E(Ep0, i, j)) / (dx / 2.0) + (E(Et, i + 1, j + 1) - E(Ep0, i, j + 1)) / (dx / 2.0));
  double t3 = 0.5 * ((E(E0p, i, j) - E(Et, i, j)) / (dy / 2.0) + (E(E0p, i + 1, j) - E(Et, i + 1, j)) / (dy / 2.0));
  double t4 = 0.5 * ((E(Et, i, j + 1) - E(E0p, i, j)) / (dy / 2.0) + (E(Et, i + 1, j + 1) - E(E0p, i + 1, j)) / (dy / 2.0));
#undef E
  return bar + dx / 8.0 * (t1 - t2) + dy / 8.0 * (t3 - t4);
}
static void cell_ez(double* Et, const double* ucon) {
  const size_t N = G.N;
  for (size_t c = 0; c < N; ++c)
    Et[c] = ucon[2 * N + c] / ucon[c] * ucon[5 * N + c] - ucon[N + c] / ucon[c] * ucon[6 * N + c];
}
/* eq (39) face update and eq (46) cell average, ct_flux.cpp:176-189.  Epp is the corner
 * grid of (nx+1)(ny+1) corners from (-1/2, -1/2): EC(i, j) = corner (i+1/2, j+1/2). */
#define EC(i, j) Epp[(size_t)((i) + 1) + (size_t)(G.nx + 1) * (size_t)((j) + 1)]
static void face_update(double* bx, double* by, const double* bxQs, const double* byQs, const double* Epp, double h,
                        double* ucon) {
  const size_t N = G.N;
  for (int j = 0; j < G.ny; j++)
    for (int i = 0; i < G.nx; i++) {
      bx[ID(i, j)] = bxQs[ID(i, j)] - h / G.dy * (EC(i, j) - EC(i, j - 1));
      by[ID(i, j)] = byQs[ID(i, j)] + h / G.dx * (EC(i, j) - EC(i - 1, j));
    }
  if (G.xclamp)
    for (int j = 0; j < G.ny; j++) bx[N + j] = bxQs[N + j] - h / G.dy * (EC(-1, j) - EC(-1, j - 1));
  if (G.yclamp)
    for (int i = 0; i < G.nx; i++) by[N + i] = byQs[N + i] + h / G.dx * (EC(i, -1) - EC(i - 1, -1));
  for (int j = 0; j < G.ny; j++)
    for (int i = 0; i < G.nx; i++) {
      ucon[5 * N + ID(i, j)] = 0.5 * (BXF(bx, i - 1, j) + bx[ID(i, j)]);
      ucon[6 * N + ID(i, j)] = 0.5 * (BYF(by, i, j - 1) + by[ID(i, j)]);
    }
}
static void corner_grid(double* Epp, const double* Ep0, const double* E0p, const double* Et) {
  for (int j = -1; j < G.ny; j++)
    for (int i = -1; i < G.nx; i++) EC(i, j) = corner_at(i, j, Ep0, E0p, Et);
}
#undef EC
/* Staggered_CT_Consistent, ct_flux.cpp:150-191 */
static void staggered_ct_consistent(double* ucon, double* bx, double* by, const double* bxQs, const double* byQs,
                                    const double* Fx, const double* Fy, double h) {
  const size_t N = G.N;
  double *Ep0 = alloc(N), *E0p = alloc(N), *Et = alloc(N), *Epp = alloc((size_t)(G.nx + 1) * (G.ny + 1));
  for (size_t c = 0; c < N; ++c) {
    Ep0[c] = -Fx[c];
    E0p[c] = +Fy[c];
  }
  cell_ez(Et, ucon);
  corner_grid(Epp, Ep0, E0p, Et);
  face_update(bx, by, bxQs, byQs, Epp, h, ucon);
  free(Ep0); free(E0p); free(Et); free(Epp);
}
/* Unstaggered_CT_Consistent, constrained_transport.cpp:500-540 */
static void unstaggered_ct_consistent(double* ucon, double* A, const double* A_s, const double* Fx, const double* Fy,
                                      double h) {
  const size_t N = G.N;
  double *Ep0 = alloc(N), *E0p = alloc(N), *Et = alloc(N), *Epp = alloc((size_t)(G.nx + 1) * (G.ny + 1));
  for (size_t c = 0; c < N; ++c) {
    Ep0[c] = -Fx[c];
    E0p[c] = +Fy[c];
  }
  cell_ez(Et, ucon);
  corner_grid(Epp, Ep0, E0p, Et);
#define EC(i, j) Epp[(size_t)((i) + 1) + (size_t)(G.nx + 1) * (size_t)((j) + 1)]
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      double Ec = 0.25 * (EC(i, j) + EC(i - 1, j) + EC(i, j - 1) + EC(i - 1, j - 1));
      A[2 * N + ID(i, j)] = A_s[2 * N + ID(i, j)] - h * Ec;
    }
#undef EC
  const double* A2 = A + 2 * N;
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      ucon[5 * N + ID(i, j)] = (agh(A2, i, j + 1) - agh(A2, i, j - 1)) / (2.0 * G.dy);
      ucon[6 * N + ID(i, j)] = -(agh(A2, i + 1, j) - agh(A2, i - 1, j)) / (2.0 * G.dx);
    }
  free(Ep0); free(E0p); free(Et); free(Epp);
}
/* Staggered_CT (legacy), constrained_transport.cpp:66-143 */
static void staggered_ct_legacy(double* ucon, double* bx, double* by, const double* bxQs, const double* byQs, double h) {
  const size_t N = G.N;
  double *w = alloc(32 * N), *Ep0 = alloc(N), *E0p = alloc(N), *Et = alloc(N);
  double* Epp = alloc((size_t)(G.nx + 1) * (G.ny + 1));
  double *wxL = w, *wxR = w + 8 * N, *wyL = w + 16 * N, *wyR = w + 24 * N;
  reconstruct(ucon, wxL, wxR, wyL, wyR);
  double QL[8], QR[8];
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      load8(wxR, ID(i, j), QL);
      load8(wxL, ID(i + 1, j), QR);
      double fL6 = QL[6] * (QL[1] / QL[0]) - (QL[2] / QL[0]) * QL[5];
      double fR6 = QR[6] * (QR[1] / QR[0]) - (QR[2] / QR[0]) * QR[5];
      Ep0[ID(i, j)] = -(0.5 * (fL6 + fR6));
      load8(wyR, ID(i, j), QL);
      load8(wyL, ID(i, j + 1), QR);
      double gL5 = QL[5] * (QL[2] / QL[0]) - (QL[1] / QL[0]) * QL[6];
      double gR5 = QR[5] * (QR[2] / QR[0]) - (QR[1] / QR[0]) * QR[6];
      E0p[ID(i, j)] = (0.5 * (gL5 + gR5));
    }
  cell_ez(Et, ucon);
  corner_grid(Epp, Ep0, E0p, Et);
  face_update(bx, by, bxQs, byQs, Epp, h, ucon);
  free(w); free(Ep0); free(E0p); free(Et); free(Epp);
}
static double vanleer_lim(double a, double b) {
  if (a * b <= 0.0) return 0.0;
  return 2.0 * a * b / (a + b);
}
/* Unstaggered_CT (legacy), constrained_transport.cpp:436-498: A_s and A are read with the
 * ghosts of bound_cond_A (constrained_transport.cpp:438,486), u_con with those of bound_cond_u */
static void unstaggered_ct_legacy(double* ucon, double* A, const double* A_s, double h) {
  const size_t N = G.N;
  const double dx = G.dx, dy = G.dy;
  const double* A2 = A + 2 * N;
#define UA(k, ii, jj) AT(ucon, k, ii, jj)
#define AS(ii, jj) agh(A_s + 2 * N, ii, jj)
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      double uL = 0.5 * (UA(1, i - 1, j) / UA(0, i - 1, j) + UA(1, i, j) / UA(0, i, j));
      double uR = 0.5 * (UA(1, i, j) / UA(0, i, j) + UA(1, i + 1, j) / UA(0, i + 1, j));
      double dAL = AS(i, j) - AS(i - 1, j), dAR = AS(i + 1, j) - AS(i, j);
      double dALL = AS(i - 1, j) - AS(i - 2, j), dARR = AS(i + 2, j) - AS(i + 1, j);
      double fluct_x = fmax(uL, 0.0) * dAL + fmin(uR, 0.0) * dAR;
      double corrL = 0.5 * fabs(uL) * (1.0 - fabs(uL) * h / dx) * vanleer_lim(dAL, (uL >= 0.0 ? dALL : dAR));
      double corrR = 0.5 * fabs(uR) * (1.0 - fabs(uR) * h / dx) * vanleer_lim(dAR, (uR >= 0.0 ? dAL : dARR));
      double dAdt_x = fluct_x / dx + (corrR - corrL) / dx;
      double vL = 0.5 * (UA(2, i, j - 1) / UA(0, i, j - 1) + UA(2, i, j) / UA(0, i, j));
      double vR = 0.5 * (UA(2, i, j) / UA(0, i, j) + UA(2, i, j + 1) / UA(0, i, j + 1));
      double dAB = AS(i, j) - AS(i, j - 1), dAT = AS(i, j + 1) - AS(i, j);
      double dABB = AS(i, j - 1) - AS(i, j - 2), dATT = AS(i, j + 2) - AS(i, j + 1);
      double fluct_y = fmax(vL, 0.0) * dAB + fmin(vR, 0.0) * dAT;
      double corrB = 0.5 * fabs(vL) * (1.0 - fabs(vL) * h / dy) * vanleer_lim(dAB, (vL >= 0.0 ? dABB : dAT));
      double corrT = 0.5 * fabs(vR) * (1.0 - fabs(vR) * h / dy) * vanleer_lim(dAT, (vR >= 0.0 ? dAB : dATT));
      double dAdt_y = fluct_y / dy + (corrT - corrB) / dy;
      A[2 * N + ID(i, j)] = AS(i, j) - h * (dAdt_x + dAdt_y);
    }
#undef UA
#undef AS
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      ucon[5 * N + ID(i, j)] = (agh(A2, i, j + 1) - agh(A2, i, j - 1)) / (2.0 * dy);
      ucon[6 * N + ID(i, j)] = -(agh(A2, i + 1, j) - agh(A2, i - 1, j)) / (2.0 * dx);
    }
}

/* ------------------------------------------------------------------ */
/* step-level scalars, timestep.cpp                                   */
/* ------------------------------------------------------------------ */
/* calch timestep.cpp:89-120 */
static void calch(void) {
  double cx = 1e-8, cy = 1e-8, cc = 1e-8, p[8];
  for (size_t n = 0; n < G.N; ++n) {
    load8(G.prim, n, p);
    double B2 = p[5] * p[5] + p[6] * p[6] + p[7] * p[7];
    double B = sqrt(B2);
    double v = sqrt(p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
    double cfx = eos_fast(p[0], p[4], p[5], B2);
    double cfy = eos_fast(p[0], p[4], p[6], B2);
    double cf = eos_fast(p[0], p[4], B, B2);
    if (cx < p[1] + cfx) cx = p[1] + cfx;
    if (cy < p[2] + cfy) cy = p[2] + cfy;
    if (cc < v + cf) cc = v + cf;
  }
  G.ch_x = cx;
  G.ch_y = cy;
  G.ch = cc;
}
/* calca timestep.cpp:122-148 */
static void calca(void) {
  double ax = 1e-8, ay = 1e-8, aa = 1e-8, p[8];
  for (size_t n = 0; n < G.N; ++n) {
    load8(G.prim, n, p);
    double B = sqrt(p[5] * p[5] + p[6] * p[6] + p[7] * p[7]);
    if (ax < p[5] / sqrt(p[0])) ax = p[5] / sqrt(p[0]);
    if (ay < p[6] / sqrt(p[0])) ay = p[6] / sqrt(p[0]);
    if (aa < B / sqrt(p[0])) aa = B / sqrt(p[0]);
  }
  G.cA_x = ax;
  G.cA_y = ay;
  G.cA = aa;
}
/* caldt timestep.cpp:5-67 */
static double caldt(void) {
  double vxm = 0, vym = 0, vm = 0;
  const size_t N = G.N;
  for (size_t n = 0; n < N; ++n) {
    double vx = G.prim[N + n], vy = G.prim[2 * N + n], vz = G.prim[3 * N + n];
    if (fabs(vx) > fabs(vxm)) vxm = fabs(vx);
    if (fabs(vy) > fabs(vym)) vym = fabs(vy);
    if (sqrt(vx * vx + vy * vy + vz * vz) > fabs(vm)) vm = sqrt(vx * vx + vy * vy + vz * vz);
  }
  G.vx_max = vxm;
  G.vy_max = vym;
  G.v_max = vm;
  int full_step = 1;
  switch (PP.caltimestep) {
    case Fullydt: G.a_max = G.ch; break;
    case Alfvendt: G.a_max = (G.timestep < full_step + 1) ? G.ch : G.cA; break;
    default: G.a_max = (G.timestep < full_step + 1) ? G.ch : vm; break;
  }
  double dt = PP.CFL * 1 / (2 * G.a_max / fmin(G.dx, G.dy));
  if (G.timestep > 1 && G.prev_dt > 0.0) dt = fmin(dt, 2.0 * G.prev_dt);
  G.prev_dt = dt;
  if (G.timestep > full_step) G.a_max = vm;
  return dt;
}
/* MagneticEigenvalues timestep.cpp:254-273 */
static void magnetic_eigenvalues(void) {
  double bx = 0, by = 0, p[8];
  for (size_t n = 0; n < G.N; ++n) {
    load8(G.prim, n, p);
    double B2 = p[5] * p[5] + p[6] * p[6] + p[7] * p[7];
    double b_x = 0.5 * (fabs(p[1]) + sqrt(p[1] * p[1] + 4 * B2 / p[0]));
    double b_y = 0.5 * (fabs(p[2]) + sqrt(p[2] * p[2] + 4 * B2 / p[0]));
    if (fabs(bx) < fabs(b_x)) bx = b_x;
    if (fabs(by) < fabs(b_y)) by = b_y;
  }
  G.B_max_x = bx;
  G.B_max_y = by;
}

/* ------------------------------------------------------------------ */
/* snapshots                                                          */
/* ------------------------------------------------------------------ */
static void keep(double** dst, const double* src, size_t n) {
  if (!*dst) *dst = alloc(n);
  memcpy(*dst, src, n * sizeof(double));
}
static void snapshot(int sub, int rks) {
  if (!G.snap_on || rks >= MAXRK) return;
  snap_t* s = &G.snaps[rks][sub];
  size_t N = G.N;
  keep(&s->u_con, G.cons, 8 * N);
  keep(&s->Qe, G.Qe, 8 * N);
  keep(&s->Qs, G.Qs, 8 * N);
  keep(&s->bx, G.bx, G.NF);
  keep(&s->by, G.by, G.NF);
  keep(&s->bxQs, G.bxQs, G.NF);
  keep(&s->byQs, G.byQs, G.NF);
  keep(&s->A, G.A, 3 * N);
  keep(&s->A_s, G.A_s, 3 * N);
  keep(&s->Fx, G.Fx, N);
  keep(&s->Fy, G.Fy, N);
  s->valid = 1;
}

/* ------------------------------------------------------------------ */
/* one IMEX stage, main.cpp:367-558                                   */
/* ------------------------------------------------------------------ */
static void stage(int rks) {
  const size_t N = G.N;
  const double dt = G.dt;
  memcpy(G.Qe, G.cons_n, 8 * N * sizeof(double));
  memcpy(G.Qs, G.cons_n, 8 * N * sizeof(double));
  memcpy(G.A_s, G.A_snap, 3 * N * sizeof(double));
  memcpy(G.A_e, G.A_snap, 3 * N * sizeof(double));
  const size_t NF = G.NF;
  memcpy(G.bxQe, G.bx_n, NF * sizeof(double));
  memcpy(G.byQe, G.by_n, NF * sizeof(double));
  memcpy(G.bxQs, G.bx_n, NF * sizeof(double));
  memcpy(G.byQs, G.by_n, NF * sizeof(double));
  for (int r = 0; r < rks; r++) {
    const double* H = G.Hs + (size_t)r * 8 * N;
    for (size_t n = 0; n < 8 * N; ++n) {
      G.Qe[n] = G.Qe[n] + G.Ae[rks][r] * dt * H[n];
      G.Qs[n] = G.Qs[n] + G.Ai[rks][r] * dt * H[n];
    }
  }
  for (int r = 0; r < rks; r++) {
    const double* HA = G.HsA + (size_t)r * 3 * N;
    const double* HB = G.HsB + (size_t)r * 2 * NF;
    for (size_t n = 0; n < 3 * N; ++n) {
      G.A_e[n] += G.Ae[rks][r] * dt * HA[n];
      G.A_s[n] += G.Ai[rks][r] * dt * HA[n];
    }
    for (size_t n = 0; n < NF; ++n) {
      G.bxQe[n] += G.Ae[rks][r] * dt * HB[n];
      G.byQe[n] += G.Ae[rks][r] * dt * HB[NF + n];
      G.bxQs[n] += G.Ai[rks][r] * dt * HB[n];
      G.byQs[n] += G.Ai[rks][r] * dt * HB[NF + n];
    }
  }
  memcpy(G.A, G.A_s, 3 * N * sizeof(double));
  G.adt = G.Ai[rks][rks] * dt;
  const double adt = G.adt;
  snapshot(SUB_COMBINE, rks);

  reconstruct(G.Qe, G.wxL, G.wxR, G.wyL, G.wyR);
  flux_update(rusanovC, G.cons, G.Qs, G.wxL, G.wxR, G.wyL, G.wyR, adt);
  snapshot(SUB_CONVECTIVE, rks);

  if (PP.magfield == PotentialA) mag_subsystem_A(G.cons, G.Qs, G.Qe, G.A, G.A_s, adt);
  else mag_subsystem_B(G.cons, G.Qs, G.Qe, adt, G.Fx, G.Fy);
  snapshot(SUB_MAGNETIC, rks);

  memcpy(G.Bsave, PL(G.cons, 5), 3 * N * sizeof(double));
  double* ws[4] = {G.wxL, G.wxR, G.wyL, G.wyR};
  for (int q = 0; q < 4; ++q) memcpy(PL(ws[q], 5), PL(G.cons, 5), 3 * N * sizeof(double));
  /* main.cpp:469-485 */
  flux_update(PP.formula == EnergyFormula ? energy_flux : pressure_flux, G.cons, G.Qs, G.wxL, G.wxR, G.wyL, G.wyR,
              adt);
  snapshot(SUB_PFLUX, rks);

  if (PP.formula == EnergyFormula) pre_subsystem_energy(G.cons, G.Qe, adt);
  else pre_subsystem_pressure(G.cons, G.Qs, G.Qe, adt, rks);
  snapshot(SUB_PRESSURE, rks);

  if (PP.magfield == StaggerCT) {
    staggered_ct_consistent(G.cons, G.bx, G.by, G.bxQs, G.byQs, G.Fx, G.Fy, adt);
    snapshot(SUB_CT, rks);
  } else if (PP.magfield == UnStaggerCT) {
    unstaggered_ct_consistent(G.cons, G.A, G.A_s, G.Fx, G.Fy, adt);
    snapshot(SUB_CT, rks);
  }
  if (PP.Energy_modify) {
    for (size_t c = 0; c < N; ++c) {
      double b5 = G.cons[5 * N + c], b6 = G.cons[6 * N + c], b7 = G.cons[7 * N + c];
      double o5 = G.Bsave[c], o6 = G.Bsave[N + c], o7 = G.Bsave[2 * N + c];
      G.cons[4 * N + c] = G.cons[4 * N + c] + ((b5 * b5 + b6 * b6 + b7 * b7) - (o5 * o5 + o6 * o6 + o7 * o7)) / 2.0;
    }
  }
  grid_con2pri(G.prim, G.cons);
  double* H = G.Hs + (size_t)rks * 8 * N;
  for (size_t n = 0; n < 8 * N; ++n) H[n] = (G.cons[n] - G.Qs[n]) / adt;
  double* HA = G.HsA + (size_t)rks * 3 * N;
  for (size_t n = 0; n < 3 * N; ++n) HA[n] = (G.A[n] - G.A_s[n]) / adt;
  double* HB = G.HsB + (size_t)rks * 2 * G.NF;
  for (size_t n = 0; n < G.NF; ++n) {
    HB[n] = (G.bx[n] - G.bxQs[n]) / adt;
    HB[G.NF + n] = (G.by[n] - G.byQs[n]) / adt;
  }
}

/* ------------------------------------------------------------------ */
/* public interface                                                   */
/* ------------------------------------------------------------------ */
static void free_all(void) {
  double** ps[] = {&G.prim, &G.cons, &G.cons_n, &G.Qe, &G.Qs, &G.wxL, &G.wxR, &G.wyL, &G.wyR, &G.bx, &G.by,
                   &G.bx_n, &G.by_n, &G.bxQe, &G.byQe, &G.bxQs, &G.byQs, &G.Fx, &G.Fy, &G.A, &G.A_s, &G.A_e,
                   &G.A_snap, &G.Hs, &G.HsA, &G.HsB, &G.Bsave};
  for (size_t i = 0; i < sizeof ps / sizeof ps[0]; ++i) {
    free(*ps[i]);
    *ps[i] = NULL;
  }
  for (int r = 0; r < MAXRK; ++r)
    for (int s = 0; s < NSUB; ++s) {
      snap_t* q = &G.snaps[r][s];
      double** qs[] = {&q->u_con, &q->Qe, &q->Qs, &q->bx, &q->by, &q->bxQs, &q->byQs, &q->A, &q->A_s, &q->Fx, &q->Fy};
      for (size_t i = 0; i < sizeof qs / sizeof qs[0]; ++i) {
        free(*qs[i]);
        *qs[i] = NULL;
      }
      q->valid = 0;
    }
  G.ready = 0;
}

int ora_setup(int nx, int ny, int rks, const ora_params* p) {
  if (nx < 4 || ny < 4 || rks < 1 || rks > MAXRK) return 1;
  if ((p->formula != PressureFormula && p->formula != EnergyFormula) ||
      (p->U_update != DefinitionofU && p->U_update != ConservationofU))
    return 2;
  free_all();
  G.nx = nx;
  G.ny = ny;
  G.R = rks;
  G.N = (size_t)nx * ny;
  G.NF = G.N + (size_t)nx + (size_t)ny;
  G.xclamp = G.yclamp = 0;
  G.P = *p;
  G.dx = (p->x1 - p->x0) / nx;
  G.dy = (p->y1 - p->y0) / ny;
  size_t N = G.N;
  G.prim = alloc(8 * N); G.cons = alloc(8 * N); G.cons_n = alloc(8 * N); G.Qe = alloc(8 * N); G.Qs = alloc(8 * N);
  G.wxL = alloc(8 * N); G.wxR = alloc(8 * N); G.wyL = alloc(8 * N); G.wyR = alloc(8 * N);
  const size_t NF = G.NF;
  G.bx = alloc(NF); G.by = alloc(NF); G.bx_n = alloc(NF); G.by_n = alloc(NF); G.bxQe = alloc(NF); G.byQe = alloc(NF);
  G.bxQs = alloc(NF); G.byQs = alloc(NF); G.Fx = alloc(N); G.Fy = alloc(N);
  G.A = alloc(3 * N); G.A_s = alloc(3 * N); G.A_e = alloc(3 * N); G.A_snap = alloc(3 * N);
  G.Hs = alloc((size_t)rks * 8 * N); G.HsA = alloc((size_t)rks * 3 * N); G.HsB = alloc((size_t)rks * 2 * NF);
  G.Bsave = alloc(3 * N);
  memset(G.Ae, 0, sizeof G.Ae);
  memset(G.Ai, 0, sizeof G.Ai);
  /* Butcher tableaux, main.cpp:269-319 */
  if (rks == 1) {
    G.Ae[0][0] = 0.0;
    G.Ai[0][0] = 1.0;
  } else if (rks == 2) {
    double bb = 1.0 - 1.0 / sqrt(2.0), cc = 1.0 / (2.0 * bb);
    G.Ae[1][0] = cc;
    G.Ai[0][0] = bb;
    G.Ai[1][0] = 1 - bb;
    G.Ai[1][1] = bb;
  } else {
    double r12 = 0.5, r13 = 1.0 / 3.0, r14 = 1.0 / 4.0;
    G.Ae[1][0] = r12;
    G.Ae[2][0] = r12;
    G.Ae[2][1] = r12;
    G.Ai[0][0] = r14;
    G.Ai[1][1] = r14;
    G.Ai[2][0] = r13;
    G.Ai[2][1] = r13;
    G.Ai[2][2] = r13;
  }
  G.t = 0;
  G.dt = 0;
  G.timestep = 0;
  G.prev_dt = 0;
  G.Mbig = 0;
  G.max_floored = 0;
  G.min_p_ever = 1e300;
  G.ready = 1;
  return 0;
}

int ora_load_prim(const double* prim8, const double* bx, const double* by, const double* A3) {
  if (!G.ready) return 1;
  size_t N = G.N;
  memcpy(G.prim, prim8, 8 * N * sizeof(double));
  memcpy(G.bx, bx, N * sizeof(double));
  memcpy(G.by, by, N * sizeof(double));
  memcpy(G.A, A3, 3 * N * sizeof(double));
  grid_pri2con(G.cons, G.prim);
  G.t = 0;
  G.timestep = 0;
  return 0;
}

/* one time step, main.cpp:335-561 */
double ora_step(int snapshots) {
  if (!G.ready) return -1.0;
  G.snap_on = snapshots;
  for (int r = 0; r < MAXRK; ++r)
    for (int s = 0; s < NSUB; ++s) G.snaps[r][s].valid = 0;
  size_t N = G.N;
  G.timestep++;
  calch();
  calca();
  double d = caldt();
  G.dt = fmin(d, PP.time_stop - G.t);
  if (PP.fixed_dt > 0.0) G.dt = fmin(PP.fixed_dt, PP.time_stop - G.t);
  memcpy(G.A_snap, G.A, 3 * N * sizeof(double));
  magnetic_eigenvalues();
  G.t = G.t + G.dt;
  grid_pri2con(G.cons, G.prim);
  memcpy(G.cons_n, G.cons, 8 * N * sizeof(double));
  memcpy(G.bx_n, G.bx, G.NF * sizeof(double));
  memcpy(G.by_n, G.by, G.NF * sizeof(double));
  for (int r = 0; r < G.R; ++r) stage(r);
  grid_con2pri(G.prim, G.cons);
  return G.dt;
}

void ora_get_cons(double* o) { memcpy(o, G.cons, 8 * G.N * sizeof(double)); }
void ora_get_prim(double* o) { memcpy(o, G.prim, 8 * G.N * sizeof(double)); }
void ora_get_faces(double* bx, double* by) {
  memcpy(bx, G.bx, G.N * sizeof(double));
  memcpy(by, G.by, G.N * sizeof(double));
}
void ora_get_A(double* A3) { memcpy(A3, G.A, 3 * G.N * sizeof(double)); }
void ora_get_Hs(int r, double* c8, double* a3, double* b2) {
  size_t N = G.N;
  memcpy(c8, G.Hs + (size_t)r * 8 * N, 8 * N * sizeof(double));
  memcpy(a3, G.HsA + (size_t)r * 3 * N, 3 * N * sizeof(double));
  memcpy(b2, G.HsB + (size_t)r * 2 * G.NF, N * sizeof(double));
  memcpy(b2 + N, G.HsB + (size_t)r * 2 * G.NF + G.NF, N * sizeof(double));
}
void ora_get_scalars(double* o) {
  o[0] = G.dt; o[1] = G.adt; o[2] = G.B_max_x; o[3] = G.B_max_y; o[4] = G.vx_max; o[5] = G.vy_max;
  o[6] = G.a_max; o[7] = G.t; o[8] = G.ch; o[9] = G.v_max; o[10] = (double)G.timestep; o[11] = G.Mbig;
  o[12] = (double)G.max_floored; o[13] = G.min_p_ever;
}
void ora_set_scalars(const double* in) {
  G.dt = in[0]; G.adt = in[1]; G.B_max_x = in[2]; G.B_max_y = in[3]; G.vx_max = in[4]; G.vy_max = in[5];
  G.a_max = in[6];
}
void ora_get_tableau(double* ae, double* ai) {
  for (int r = 0; r < G.R; ++r)
    for (int c = 0; c < G.R; ++c) {
      ae[r * G.R + c] = G.Ae[r][c];
      ai[r * G.R + c] = G.Ai[r][c];
    }
}
int ora_get_snapshot(int rks, int sub, int which, double* out) {
  if (rks < 0 || rks >= MAXRK || sub < 0 || sub >= NSUB) return 1;
  snap_t* s = &G.snaps[rks][sub];
  if (!s->valid) return 2;
  size_t N = G.N;
  switch (which) {
    case 0: memcpy(out, s->u_con, 8 * N * sizeof(double)); break;
    case 1: memcpy(out, s->Qe, 8 * N * sizeof(double)); break;
    case 2: memcpy(out, s->Qs, 8 * N * sizeof(double)); break;
    case 3: memcpy(out, s->bx, N * sizeof(double)); break;
    case 4: memcpy(out, s->by, N * sizeof(double)); break;
    case 5: memcpy(out, s->bxQs, N * sizeof(double)); break;
    case 6: memcpy(out, s->byQs, N * sizeof(double)); break;
    case 7: memcpy(out, s->A, 3 * N * sizeof(double)); break;
    case 8: memcpy(out, s->A_s, 3 * N * sizeof(double)); break;
    case 9: memcpy(out, s->Fx, N * sizeof(double)); break;
    case 10: memcpy(out, s->Fy, N * sizeof(double)); break;
    default: return 3;
  }
  return 0;
}

void ora_fn_reconstruct(const double* Q8, double* out32) {
  size_t N = G.N;
  reconstruct(Q8, out32, out32 + 8 * N, out32 + 16 * N, out32 + 24 * N);
}
void ora_fn_shock(const double* Q8, double* eta) { shock_detector(eta, Q8); }

void ora_fn_operator(int op, const double* ucon8, const double* Qe8, const double* Qs8, double h,
                     const double* pfreeze, double mbig, const double* x, double* Ax) {
  if (op == 0 || op == 1) {
    pressure_setup(ucon8, Qe8, Qs8, h);
    OP.jac = op == 1;
    OP.pfreeze = (double*)pfreeze;
    if (op == 1) G.Mbig = mbig;
    pressure_ax(x, Ax);
    OP.jac = 0;
    OP.pfreeze = NULL;
  } else if (op == 2) {
    OP.ucon = ucon8;
    OP.Qe = Qe8;
    OP.Qs = Qs8;
    OP.h = h;
    magnetic_ax(x, Ax);
  } else if (op == 3) {
    OP.ucon = ucon8;
    OP.Qe = Qe8;
    OP.Qs = Qs8;
    OP.h = h;
    potential_gmax(Qs8);
    potential_ax(x, Ax);
  } else if (op == 4) {
    energy_setup(ucon8, Qe8, h);
    energy_ax(x, Ax);
  }
}

void ora_fn_nested_newton(const double* ucon8, const double* Qe8, const double* Qs8, double h, const double* b,
                          double* p) {
  pressure_setup(ucon8, Qe8, Qs8, h);
  nested_newton(p, b);
}

void ora_fn_substep(int sub, double h, int rks, double* ucon8, const double* Qe8, const double* Qs8, double* bx,
                    double* by, const double* bxQs, const double* byQs, double* A3, const double* As3, double* Fx,
                    double* Fy) {
  size_t N = G.N;
  switch (sub) {
    case 1:
      reconstruct(Qe8, G.wxL, G.wxR, G.wyL, G.wyR);
      flux_update(rusanovC, ucon8, Qs8, G.wxL, G.wxR, G.wyL, G.wyR, h);
      break;
    case 2:
      if (PP.magfield == PotentialA) mag_subsystem_A(ucon8, Qs8, Qe8, A3, As3, h);
      else mag_subsystem_B(ucon8, Qs8, Qe8, h, Fx, Fy);
      break;
    case 3: {
      reconstruct(Qe8, G.wxL, G.wxR, G.wyL, G.wyR);
      double* ws[4] = {G.wxL, G.wxR, G.wyL, G.wyR};
      for (int q = 0; q < 4; ++q) memcpy(PL(ws[q], 5), PL(ucon8, 5), 3 * N * sizeof(double));
      flux_update(PP.formula == EnergyFormula ? energy_flux : pressure_flux, ucon8, Qs8, G.wxL, G.wxR, G.wyL, G.wyR,
                  h);
      break;
    }
    case 4:
      if (PP.formula == EnergyFormula) pre_subsystem_energy(ucon8, Qe8, h);
      else pre_subsystem_pressure(ucon8, Qs8, Qe8, h, rks);
      break;
    case 5:
    case 6: {
      /* the caller's face planes are interior-only; the boundary lines of a transmissive
       * direction come from (and go back to) the solver's own face arrays */
      const size_t NF = G.NF, L = NF - N;
      double *fx = alloc(NF), *fy = alloc(NF), *fxs = alloc(NF), *fys = alloc(NF);
      memcpy(fx, bx, N * sizeof(double)); memcpy(fx + N, G.bx + N, L * sizeof(double));
      memcpy(fy, by, N * sizeof(double)); memcpy(fy + N, G.by + N, L * sizeof(double));
      memcpy(fxs, bxQs, N * sizeof(double)); memcpy(fxs + N, G.bxQs + N, L * sizeof(double));
      memcpy(fys, byQs, N * sizeof(double)); memcpy(fys + N, G.byQs + N, L * sizeof(double));
      if (sub == 5) {
        if (PP.magfield == StaggerCT) staggered_ct_consistent(ucon8, fx, fy, fxs, fys, Fx, Fy, h);
        else if (PP.magfield == UnStaggerCT) unstaggered_ct_consistent(ucon8, A3, As3, Fx, Fy, h);
      } else {
        if (PP.magfield == StaggerCT) staggered_ct_legacy(ucon8, fx, fy, fxs, fys, h);
        else if (PP.magfield == UnStaggerCT) unstaggered_ct_legacy(ucon8, A3, As3, h);
      }
      memcpy(bx, fx, N * sizeof(double)); memcpy(G.bx + N, fx + N, L * sizeof(double));
      memcpy(by, fy, N * sizeof(double)); memcpy(G.by + N, fy + N, L * sizeof(double));
      free(fx); free(fy); free(fxs); free(fys);
      break;
    }
    default:
      break;
  }
}

/* cal_divergence_error, imex_subsystems.cpp:630-660 */
double ora_div_error(void) {
  double err = 0;
  size_t N = G.N;
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      double d;
      if (PP.magfield == StaggerCT) {
        d = (G.bx[ID(i, j)] - BXF(G.bx, i - 1, j)) / G.dx + (G.by[ID(i, j)] - BYF(G.by, i, j - 1)) / G.dy;
      } else {
        double dBxdx, dBydy;
        const double* B5 = G.cons + 5 * N;
        const double* B6 = G.cons + 6 * N;
        if (i == 0) dBxdx = (B5[ID(i + 1, j)] - B5[ID(i, j)]) / G.dx;
        else if (i == G.nx - 1) dBxdx = (B5[ID(i, j)] - B5[ID(i - 1, j)]) / G.dx;
        else dBxdx = (B5[ID(i + 1, j)] - B5[ID(i - 1, j)]) / (2.0 * G.dx);
        if (j == 0) dBydy = (B6[ID(i, j + 1)] - B6[ID(i, j)]) / G.dy;
        else if (j == G.ny - 1) dBydy = (B6[ID(i, j)] - B6[ID(i, j - 1)]) / G.dy;
        else dBydy = (B6[ID(i, j + 1)] - B6[ID(i, j - 1)]) / (2.0 * G.dy);
        d = dBxdx + dBydy;
      }
      err += G.dx * G.dy * d * d;
    }
  return sqrt(err);
}

/* Boundary conditions per direction (config.hpp:36-37 ordinals): 0 Transmissive or
 * 2 Periodic.  Call after ora_setup and before ora_load_prim.  Every magnetic form runs
 * with either, the legacy CT variants (fn_substep 6) included. */
int ora_set_bc(int x_bc, int y_bc) {
  if (!G.ready) return 1;
  if ((x_bc != 0 && x_bc != 2) || (y_bc != 0 && y_bc != 2)) return 2;
  G.xclamp = x_bc == 0;
  G.yclamp = y_bc == 0;
  return 0;
}
/* boundary normal faces: Bx on x = x_0 (ny values), By on y = y_0 (nx values) */
void ora_set_boundary_faces(const double* bx_x0, const double* by_y0) {
  memcpy(G.bx + G.N, bx_x0, (size_t)G.ny * sizeof(double));
  memcpy(G.by + G.N, by_y0, (size_t)G.nx * sizeof(double));
}
/* a periodic direction reports the face it identifies with x_0 / y_0 (the one at x_1 / y_1) */
static void boundary_lines(const double* bxa, const double* bya, double* bx_x0, double* by_y0) {
  if (bx_x0)
    for (int j = 0; j < G.ny; ++j) bx_x0[j] = BXF(bxa, -1, j);
  if (by_y0)
    for (int i = 0; i < G.nx; ++i) by_y0[i] = BYF(bya, i, -1);
}
void ora_get_boundary_faces(double* bx_x0, double* by_y0) { boundary_lines(G.bx, G.by, bx_x0, by_y0); }
int ora_get_snapshot_boundary(int rks, int sub, int which, double* out) {
  if (rks < 0 || rks >= MAXRK || sub < 0 || sub >= NSUB) return 1;
  snap_t* s = &G.snaps[rks][sub];
  if (!s->valid) return 2;
  const double* v = which == 3 ? s->bx : which == 4 ? s->by : which == 5 ? s->bxQs : which == 6 ? s->byQs : NULL;
  if (!v) return 3;
  if (which == 3 || which == 5) boundary_lines(v, NULL, out, NULL);
  else boundary_lines(NULL, v, NULL, out);
  return 0;
}

/* Diagnose_CT_EMF with CT_EMF_Stats, constrained_transport.cpp:166-222 (printed by the
 * reference's driver after every step, main.cpp:594): the statistics it prints, returned.
 * out[4 c + q]: c = central, rusanov, tilde, total; q = L2(Ez), max|Ez|, L2(dB/dt), max|dB/dt|. */
void ora_ct_diag(double* out) {
  const size_t N = G.N;
  const double dx = G.dx, dy = G.dy;
  double* w = alloc(32 * N);
  double *cp0 = alloc(N), *c0p = alloc(N), *rp0 = alloc(N), *r0p = alloc(N), *zero = alloc(N), *et = alloc(N);
  double *wxL = w, *wxR = w + 8 * N, *wyL = w + 16 * N, *wyR = w + 24 * N;
  reconstruct(G.cons, wxL, wxR, wyL, wyR);
  double QL[8], QR[8];
  for (int i = 0; i < G.nx; i++)
    for (int j = 0; j < G.ny; j++) {
      const size_t c = ID(i, j);
      load8(wxR, c, QL);
      load8(wxL, ID(i + 1, j), QR);
      double fL6 = QL[6] * (QL[1] / QL[0]) - (QL[2] / QL[0]) * QL[5];
      double fR6 = QR[6] * (QR[1] / QR[0]) - (QR[2] / QR[0]) * QR[5];
      cp0[c] = -(0.5 * (fL6 + fR6));
      rp0[c] = 0.5 * fmax(fabs(QL[1] / QL[0]), fabs(QR[1] / QR[0])) * (QR[6] - QL[6]);
      load8(wyR, c, QL);
      load8(wyL, ID(i, j + 1), QR);
      double gL5 = QL[5] * (QL[2] / QL[0]) - (QL[1] / QL[0]) * QL[6];
      double gR5 = QR[5] * (QR[2] / QR[0]) - (QR[1] / QR[0]) * QR[6];
      c0p[c] = 0.5 * (gL5 + gR5);
      r0p[c] = -0.5 * fmax(fabs(QL[2] / QL[0]), fabs(QR[2] / QR[0])) * (QR[5] - QL[5]);
    }
  cell_ez(et, G.cons);
  const double* ep[3] = {cp0, rp0, zero};
  const double* eq[3] = {c0p, r0p, zero};
  const double* tt[3] = {zero, zero, et};
  double l2E[4] = {0, 0, 0, 0}, mxE[4] = {0, 0, 0, 0}, l2B[4] = {0, 0, 0, 0}, mxB[4] = {0, 0, 0, 0};
  for (int j = 0; j < G.ny; j++)
    for (int i = 0; i < G.nx; i++) {
      double e[4][3];
      for (int k = 0; k < 3; ++k) {
        e[k][0] = corner_at(i, j, ep[k], eq[k], tt[k]);
        e[k][1] = corner_at(i, j - 1, ep[k], eq[k], tt[k]);
        e[k][2] = corner_at(i - 1, j, ep[k], eq[k], tt[k]);
      }
      for (int q = 0; q < 3; ++q) e[3][q] = e[0][q] + e[1][q] + e[2][q];
      for (int k = 0; k < 4; ++k) {
        double v = e[k][0];
        l2E[k] += dx * dy * v * v;
        if (fabs(v) > mxE[k]) mxE[k] = fabs(v);
        double dBx = -(e[k][0] - e[k][1]) / dy;
        double dBy = (e[k][0] - e[k][2]) / dx;
        double m2 = dBx * dBx + dBy * dBy;
        l2B[k] += dx * dy * m2;
        if (sqrt(m2) > mxB[k]) mxB[k] = sqrt(m2);
      }
    }
  for (int k = 0; k < 4; ++k) {
    out[4 * k + 0] = sqrt(l2E[k]);
    out[4 * k + 1] = mxE[k];
    out[4 * k + 2] = sqrt(l2B[k]);
    out[4 * k + 3] = mxB[k];
  }
  free(w); free(cp0); free(c0p); free(rp0); free(r0p); free(zero); free(et);
}
