// Per-cell physics shared by the kernels: EOS, con<->prim, reconstruction
// stencils, explicit fluxes.  Expressions keep the reference's operand order
// (and the library is built without FMA contraction), so the explicit
// sub-steps reproduce the reference bit for bit in FP64.
#pragma once

#include <cuda_runtime.h>

#include "dual.cuh"
#include "imex_internal.h"

namespace imex {

// Set when a per-cell EOS Newton iteration hits its cap; one copy per translation
// unit, read and cleared by the host through eos_flag_stage / eos_flag_solve.
static __device__ int d_eos_flag = 0;

constexpr int kEosNewtonCap = 200;

__device__ __forceinline__ int wrap(int i, int n) {
  i %= n;
  return i < 0 ? i + n : i;
}
// the cell a neighbour index (|offset| < n) reads: the periodic image, or the nearest
// interior cell of a transmissive direction
__device__ __forceinline__ int cix(const DevParams& P, int i) {
  return i < 0 ? i * P.xm + P.xlo : (i >= P.nx ? i * P.xm + P.xhi : i);
}
__device__ __forceinline__ int cjy(const DevParams& P, int j) {
  return j < 0 ? j * P.ym + P.ylo : (j >= P.ny ? j * P.ym + P.yhi : j);
}
__device__ __forceinline__ long long cid(const DevParams& P, int i, int j) {
  return (long long)cix(P, i) + (long long)P.nx * cjy(P, j);
}
// the cell (i, j) of linear index n = i + nx j (n < 2^31): j = floor(n / nx) by the
// multiply-high of the invariant-divisor method (DevParams::nx_magic), no integer division
__device__ __forceinline__ void cell_of(const DevParams& P, long long n, int& i, int& j) {
  const unsigned u = (unsigned)n;
  const unsigned t = __umulhi(P.nx_magic, u);
  const unsigned q = (t + ((u - t) >> P.nx_sh1)) >> P.nx_sh2;
  j = (int)q;
  i = (int)(u - q * (unsigned)P.nx);
}
// Order key of a double: unsigned comparison of keys is numeric comparison of the values.
__device__ __forceinline__ unsigned long long dkey(double d) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(d);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double dkey_value(unsigned long long k) {
  return __longlong_as_double((long long)((k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k));
}

// The parameters a kernel instantiated for periodic (kOpen = false) or transmissive
// (kOpen = true) neighbour maps works with: the periodic instance has the wrap as
// compile-time constants, so its index arithmetic is the plain wrap.
template <bool kOpen>
__device__ __forceinline__ DevParams bc_params(const DevParams& P) {
  DevParams Q = P;
  if (!kOpen) {
    Q.xclamp = Q.yclamp = 0;
    Q.xm = Q.ym = 1;
    Q.xlo = P.nx;
    Q.xhi = -P.nx;
    Q.ylo = P.ny;
    Q.yhi = -P.ny;
  }
  return Q;
}
// Plane a of A at (i, j) with the ghosts of bound_cond_A (boundary.cpp:177-292): a
// transmissive direction extrapolates linearly from its two nearest interior cells, x first
// and then y on the x-extrapolated rows; a periodic direction wraps.
__device__ __forceinline__ double a_row(const DevParams& P, const double* __restrict__ a, int i, int j) {
  const double* r = a + (long long)P.nx * j;
  if (P.xclamp && i < 0) {
    const double slope = r[1] - r[0];
    return r[0] - (double)(-i) * slope;
  }
  if (P.xclamp && i >= P.nx) {
    const double slope = r[P.nx - 1] - r[P.nx - 2];
    return r[P.nx - 1] + (double)(i - P.nx + 1) * slope;
  }
  return r[cix(P, i)];
}
__device__ __forceinline__ double a_ghost(const DevParams& P, const double* __restrict__ a, int i, int j) {
  if (!P.xclamp && !P.yclamp) return a[cid(P, i, j)];
  if (P.yclamp && j < 0) {
    const double a0 = a_row(P, a, i, 0), slope = a_row(P, a, i, 1) - a0;
    return a0 - (double)(-j) * slope;
  }
  if (P.yclamp && j >= P.ny) {
    const double aT = a_row(P, a, i, P.ny - 1), slope = aT - a_row(P, a, i, P.ny - 2);
    return aT + (double)(j - P.ny + 1) * slope;
  }
  return a_row(P, a, i, cjy(P, j));
}

// ---------------------------------------------------------------- EOS
// The per-cell physics below is templated on its scalar type S: double in the
// forward kernels (the operations and their order are the reference's), Dual<L>
// (dual.cuh) when the adjoint differentiates a cell function.
// Redlich-Kwong thermal/caloric EOS and its Newton inversions, config.hpp:130-173.
template <class S>
__device__ inline S rk_T_from_rho_p(const DevParams& P, S rho, S p) {
  const S v = 1.0 / rho;
  S T_old, T_new = (1.0 / rho - P.m_b) * (p + P.m_alfa * rho * rho) / P.m_R;
  int it = 0;
  do {
    T_old = T_new;
    S f = P.m_R * T_old / (v - P.m_b) - P.m_alfa / sqrt(T_old) / v / (v + P.m_b) - p;
    S df = P.m_R / (v - P.m_b) + 0.5 * P.m_alfa / T_old / sqrt(T_old) / v / (v + P.m_b);
    T_new = T_old - f / df;
  } while (fabs(T_new - T_old) / fabs(T_old) > 1e-14 && ++it < kEosNewtonCap);
  if (it >= kEosNewtonCap) d_eos_flag = 1;
  return T_new;
}
template <class S>
__device__ inline S rk_e_from_rho_p(const DevParams& P, S rho, S p) {
  const S v = 1.0 / rho;
  S T = rk_T_from_rho_p(P, rho, p);
  S U = log(v / (v + P.m_b));
  return P.m_cv * T + 1.5 * P.m_alfa / P.m_b * U / sqrt(T);
}
template <class S>
__device__ inline S rk_p_from_rho_e(const DevParams& P, S rho, S e) {
  const S v = 1.0 / rho;
  S T_old, T_new = (e + rho * P.m_alfa) / P.m_cv;
  int it = 0;
  const S U = log(v / (v + P.m_b));
  do {
    T_old = T_new;
    S f = P.m_cv * T_old + 1.5 * P.m_alfa / P.m_b * U / sqrt(T_old) - e;
    S df = P.m_cv - 0.75 * P.m_alfa / P.m_b * U / T_old / sqrt(T_old);
    T_new = T_old - f / df;
  } while (fabs(T_new - T_old) / fabs(T_old) > 1e-14 && ++it < kEosNewtonCap);
  if (it >= kEosNewtonCap) d_eos_flag = 1;
  S a = P.m_alfa / sqrt(T_new);
  return P.m_R * T_new / (v - P.m_b) - a / v / (v + P.m_b);
}
template <class S>
__device__ inline S rk_sound(const DevParams& P, S rho, S p) {
  const S v = 1.0 / rho;
  S T = rk_T_from_rho_p(P, rho, p);
  S U = log(v / (v + P.m_b));
  S p_T = P.m_R / (v - P.m_b) + P.m_alfa / (2.0 * T * sqrt(T) * v * (v + P.m_b));
  S e_T = P.m_cv - 0.75 * P.m_alfa / P.m_b * U / (T * sqrt(T));
  S vmb = v - P.m_b, vpb = v + P.m_b;
  S p_v = -P.m_R * T / (vmb * vmb) + P.m_alfa * (2.0 * v + P.m_b) / (sqrt(T) * v * v * (vpb * vpb));
  S e_v = 1.5 * P.m_alfa / P.m_b * (1.0 / v - 1.0 / (v + P.m_b)) / sqrt(T);
  S a2 = p / (rho * rho) * (p_T / e_T) + v * v * (e_v - e_T * (p_v / p_T));
  return sqrt(a2);
}
// unified EOS interface, config.hpp:176-198
template <class S>
__device__ __forceinline__ S eos_p(const DevParams& P, S rho, S e) {
  return P.eos_type == IMEX_IDEAL_GAS ? (P.gamma - 1.0) * rho * e : rk_p_from_rho_e(P, rho, e);
}
template <class S>
__device__ __forceinline__ S eos_e(const DevParams& P, S rho, S p) {
  return P.eos_type == IMEX_IDEAL_GAS ? p / ((P.gamma - 1.0) * rho) : rk_e_from_rho_p(P, rho, p);
}
template <class S>
__device__ __forceinline__ S eos_a2(const DevParams& P, S rho, S p) {
  S a = P.eos_type == IMEX_IDEAL_GAS ? sqrt(P.gamma * p / rho) : rk_sound(P, rho, p);
  return a * a;
}
template <class S>
__device__ __forceinline__ S eos_fast(const DevParams& P, S rho, S p, S Bn, S B2) {
  S a2 = eos_a2(P, rho, p);
  S t = a2 + B2 / rho;
  S disc = t * t - 4.0 * a2 * Bn * Bn / rho;
  if (disc < 0) disc = 0;
  return sqrt(0.5 * (t + sqrt(disc)));
}
// V(p) = rho e(rho, p) and its slopes, config.hpp:206-239
template <class S>
__device__ __forceinline__ S Vbase(const DevParams& P, S p, S rho) {
  return P.eos_type == IMEX_IDEAL_GAS ? p / (P.gamma - 1.0) : rho * rk_e_from_rho_p(P, rho, p);
}
template <class S>
__device__ __forceinline__ S Vbase_slope(const DevParams& P, S p, S rho) {
  if (P.eos_type == IMEX_IDEAL_GAS) return S(1.0 / (P.gamma - 1.0));
  const double d = 1e-8;
  S ep = rk_e_from_rho_p(P, rho, p + d);
  S em = rk_e_from_rho_p(P, rho, p - d);
  return rho * (ep - em) / (2.0 * d);
}
template <class S>
__device__ __forceinline__ S V_mod(const DevParams& P, double Mbig, S p, S rho) {
  if (!P.floor_on) return Vbase(P, p, rho);
  return (p >= P.p_floor) ? Vbase(P, p, rho) : Vbase(P, S(P.p_floor), rho) + Mbig * (p - P.p_floor);
}
template <class S>
__device__ __forceinline__ S V_slope(const DevParams& P, double Mbig, S p, S rho) {
  if (!P.floor_on) return Vbase_slope(P, p, rho);
  return (p >= P.p_floor) ? Vbase_slope(P, p, rho) : S(Mbig);
}

// ---------------------------------------------------------------- state
// specific internal energy of a conserved state, reconstruction.cpp:291-304
template <class S>
__device__ __forceinline__ S calecon(const S* c) {
  S rho = c[0], vx = c[1] / c[0], vy = c[2] / c[0], vz = c[3] / c[0];
  S B2 = c[5] * c[5] + c[6] * c[6] + c[7] * c[7];
  S v2 = vx * vx + vy * vy + vz * vz;
  return (c[4] - 0.5 * rho * v2 - 0.5 * B2) / rho;
}
// ini_con2pri, state.cpp:206-218
template <class S>
__device__ __forceinline__ void con2pri(const DevParams& P, S* pri, const S* con) {
  S e = calecon(con);
  pri[0] = con[0];
  pri[1] = con[1] / con[0];
  pri[2] = con[2] / con[0];
  pri[3] = con[3] / con[0];
  pri[4] = eos_p(P, con[0], e);
  pri[5] = con[5];
  pri[6] = con[6];
  pri[7] = con[7];
}
// pressure of a conserved state (pri[4] of con2pri)
template <class S>
__device__ __forceinline__ S pressure_of(const DevParams& P, const S* con) {
  return eos_p(P, con[0], calecon(con));
}
// ini_pri2con, state.cpp:220-240
template <class S>
__device__ __forceinline__ void pri2con(const DevParams& P, S* con, const S* pri) {
  S e = eos_e(P, pri[0], pri[4]);
  S B2 = pri[5] * pri[5] + pri[6] * pri[6] + pri[7] * pri[7];
  S v2 = pri[1] * pri[1] + pri[2] * pri[2] + pri[3] * pri[3];
  S r = pri[0];
  con[0] = r;
  con[1] = r * pri[1];
  con[2] = r * pri[2];
  con[3] = r * pri[3];
  con[4] = r * e + 0.5 * r * v2 + 0.5 * B2;
  con[5] = pri[5];
  con[6] = pri[6];
  con[7] = pri[7];
}
// calenthalpy, timestep.cpp:224-230: e + p / rho
template <class S>
__device__ __forceinline__ S calenthalpy(const DevParams& P, const S* c) {
  S e = calecon(c);
  S p = eos_p(P, c[0], e);
  return e + p / c[0];
}
// calkinetic, timestep.cpp:239-247
template <class S>
__device__ __forceinline__ S calkinetic(const S* c) {
  S rho = c[0], vx = c[1] / c[0], vy = c[2] / c[0], vz = c[3] / c[0];
  return 0.5 * rho * (vx * vx + vy * vy + vz * vz);
}

template <int NV>
__device__ __forceinline__ void load_cell(const double* __restrict__ a, long long N, long long idx, double* o) {
#pragma unroll
  for (int k = 0; k < NV; ++k) o[k] = __ldg(a + (long long)k * N + idx);
}

// ---------------------------------------------------------------- reconstruction
// One variable along one direction from the 5-point stencil (um2 .. up2):
// left and right face values of the cell, reconstruction.cpp:38-266.
// kFast (imex_config.arith = fast): WENO5 forms its normalised weights with one division per
// face (w_k / sum w = d_k P_k / sum_i d_i P_i, P_k the product of the other two smoothness
// terms) and its polynomials with fused multiply-adds; VanLeer takes 1 / (1 + r) once.
template <class S>
__device__ inline void weno5_fast(S um2, S um1, S u0, S up1, S up2, S& wL, S& wR) {
  const S a0 = um2 - 2 * um1 + u0, b0 = fma(S(3), u0, um2 - 4 * um1);
  const S a1 = um1 - 2 * u0 + up1, b1 = um1 - up1;
  const S a2 = u0 - 2 * up1 + up2, b2 = fma(S(3), u0, up2 - 4 * up1);
  const S e0 = fma(13.0 / 12.0 * a0, a0, fma(0.25 * b0, b0, S(1e-6)));
  const S e1 = fma(13.0 / 12.0 * a1, a1, fma(0.25 * b1, b1, S(1e-6)));
  const S e2 = fma(13.0 / 12.0 * a2, a2, fma(0.25 * b2, b2, S(1e-6)));
  const S s0 = e0 * e0, s1 = e1 * e1, s2 = e2 * e2;
  const S t0 = s1 * s2, t1 = s0 * s2, t2 = s0 * s1;
  {
    const S q0 = fma(-1.0 / 6.0, um2, fma(5.0 / 6.0, um1, 1.0 / 3.0 * u0));
    const S q1 = fma(1.0 / 3.0, um1, fma(5.0 / 6.0, u0, -1.0 / 6.0 * up1));
    const S q2 = fma(11.0 / 6.0, u0, fma(-7.0 / 6.0, up1, 1.0 / 3.0 * up2));
    const S a = 0.3 * t0, b = 0.6 * t1, c = 0.1 * t2;
    wL = fma(a, q0, fma(b, q1, c * q2)) / (a + b + c);
  }
  {
    const S q0 = fma(1.0 / 3.0, um2, fma(-7.0 / 6.0, um1, 11.0 / 6.0 * u0));
    const S q1 = fma(-1.0 / 6.0, um1, fma(5.0 / 6.0, u0, 1.0 / 3.0 * up1));
    const S q2 = fma(1.0 / 3.0, u0, fma(5.0 / 6.0, up1, -1.0 / 6.0 * up2));
    const S a = 0.1 * t0, b = 0.6 * t1, c = 0.3 * t2;
    wR = fma(a, q0, fma(b, q1, c * q2)) / (a + b + c);
  }
}
// The fast WENO5 of one cell in x and y at once: the same weights and polynomials as
// weno5_fast, with the four normalisations (1 / (a + b + c) of each face) taken from one
// division of their product (plus nine multiplications) instead of four divisions.  Where
// that product leaves the normal double range (smoothness sums beyond ~1e75 or below ~1e-75)
// the four divisions are taken as in weno5_fast.
__device__ inline void weno5_fast_xy(const double (&v)[5], const double (&u)[5], double& xl, double& xr, double& yl,
                                     double& yr) {
  double nL[2], dL[2], nR[2], dR[2];
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    const double um2 = d ? u[0] : v[0], um1 = d ? u[1] : v[1], u0 = d ? u[2] : v[2];
    const double up1 = d ? u[3] : v[3], up2 = d ? u[4] : v[4];
    const double a0 = um2 - 2 * um1 + u0, b0 = fma(3.0, u0, um2 - 4 * um1);
    const double a1 = um1 - 2 * u0 + up1, b1 = um1 - up1;
    const double a2 = u0 - 2 * up1 + up2, b2 = fma(3.0, u0, up2 - 4 * up1);
    const double e0 = fma(13.0 / 12.0 * a0, a0, fma(0.25 * b0, b0, 1e-6));
    const double e1 = fma(13.0 / 12.0 * a1, a1, fma(0.25 * b1, b1, 1e-6));
    const double e2 = fma(13.0 / 12.0 * a2, a2, fma(0.25 * b2, b2, 1e-6));
    const double s0 = e0 * e0, s1 = e1 * e1, s2 = e2 * e2;
    const double t0 = s1 * s2, t1 = s0 * s2, t2 = s0 * s1;
    {
      const double q0 = fma(-1.0 / 6.0, um2, fma(5.0 / 6.0, um1, 1.0 / 3.0 * u0));
      const double q1 = fma(1.0 / 3.0, um1, fma(5.0 / 6.0, u0, -1.0 / 6.0 * up1));
      const double q2 = fma(11.0 / 6.0, u0, fma(-7.0 / 6.0, up1, 1.0 / 3.0 * up2));
      const double a = 0.3 * t0, b = 0.6 * t1, c = 0.1 * t2;
      nL[d] = fma(a, q0, fma(b, q1, c * q2));
      dL[d] = a + b + c;
    }
    {
      const double q0 = fma(1.0 / 3.0, um2, fma(-7.0 / 6.0, um1, 11.0 / 6.0 * u0));
      const double q1 = fma(-1.0 / 6.0, um1, fma(5.0 / 6.0, u0, 1.0 / 3.0 * up1));
      const double q2 = fma(1.0 / 3.0, u0, fma(5.0 / 6.0, up1, -1.0 / 6.0 * up2));
      const double a = 0.1 * t0, b = 0.6 * t1, c = 0.3 * t2;
      nR[d] = fma(a, q0, fma(b, q1, c * q2));
      dR[d] = a + b + c;
    }
  }
  const double px = dL[0] * dR[0], py = dL[1] * dR[1], pp = px * py;
  if (pp > 1e-300 && pp < 1e300) {
    const double r = 1.0 / pp;
    const double rx = py * r, ry = px * r;  // 1 / px and 1 / py
    xl = nL[0] * (dR[0] * rx);
    xr = nR[0] * (dL[0] * rx);
    yl = nL[1] * (dR[1] * ry);
    yr = nR[1] * (dL[1] * ry);
  } else {
    xl = nL[0] / dL[0];
    xr = nR[0] / dR[0];
    yl = nL[1] / dL[1];
    yr = nR[1] / dR[1];
  }
}
template <bool kFast = false, class S>
__device__ inline void recon_1d(int scheme, S um2, S um1, S u0, S up1, S up2, S& wL, S& wR, bool vortex_central) {
  S sR = up1 - u0, sL = u0 - um1, c = 0.0;
  if constexpr (kFast) {
    if (scheme == IMEX_WENO5) {
      weno5_fast(um2, um1, u0, up1, up2, wL, wR);
      return;
    }
    if (scheme == IMEX_VanLeer) {
      if (fabs(sR) < 1e-16) c = 0;
      else {
        const S r = sL / sR;
        c = (r < 0) ? S(0.0) : 2 * fmin(S(1), r) / (1 + r);
      }
      wL = fma(-0.5 * c, sL, u0);
      wR = fma(0.5 * c, sR, u0);
      return;
    }
  }
  switch (scheme) {
    case IMEX_NoRecon:
      wL = u0;
      wR = u0;
      break;
    case IMEX_Minmod:
      if (sL * sR <= 0) c = 0;
      else if (fabs(sR) <= fabs(sL)) c = sR;
      else if (fabs(sL) < fabs(sR)) c = sL;
      if (vortex_central) c = 0.5 * (sL + sR);
      wL = u0 - 0.5 * c;
      wR = u0 + 0.5 * c;
      break;
    case IMEX_VanLeer:
      if (fabs(sR) < 1e-16) c = 0;
      else {
        S r = sL / sR;
        c = (r < 0) ? S(0.0) : fmin(2 / (1 + r), (2 * r) / (1 + r));
      }
      wL = u0 - 0.5 * c * sL;
      wR = u0 + 0.5 * c * sR;
      break;
    case IMEX_ENO3: {
      S q0L = -1.0 / 6.0 * um2 + 5.0 / 6.0 * um1 + 1.0 / 3.0 * u0;
      S q1L = 1.0 / 3.0 * um1 + 5.0 / 6.0 * u0 - 1.0 / 6.0 * up1;
      S q2L = 11.0 / 6.0 * u0 - 7.0 / 6.0 * up1 + 1.0 / 3.0 * up2;
      S q0R = 1.0 / 3.0 * um2 - 7.0 / 6.0 * um1 + 11.0 / 6.0 * u0;
      S q1R = -1.0 / 6.0 * um1 + 5.0 / 6.0 * u0 + 1.0 / 3.0 * up1;
      S q2R = 1.0 / 3.0 * u0 + 5.0 / 6.0 * up1 - 1.0 / 6.0 * up2;
      S d1 = fabs(u0 - um1), d2 = fabs(up1 - u0);
      if (d1 >= d2) {
        S d3 = fabs(fabs(up2 - up1) - fabs(up1 - u0));
        S d4 = fabs(fabs(up1 - u0) - fabs(u0 - um1));
        if (d3 >= d4) { wL = q1L; wR = q1R; } else { wL = q2L; wR = q2R; }
      } else {
        S d3 = fabs(fabs(u0 - um1) - fabs(um1 - um2));
        S d4 = fabs(fabs(up1 - u0) - fabs(u0 - um1));
        if (d4 >= d3) { wL = q0L; wR = q0R; } else { wL = q1L; wR = q1R; }
      }
      break;
    }
    default: {  // WENO5
      S a0 = um2 - 2 * um1 + u0, b0 = um2 - 4 * um1 + 3 * u0;
      S a1 = um1 - 2 * u0 + up1, b1 = um1 - up1;
      S a2 = u0 - 2 * up1 + up2, b2 = 3 * u0 - 4 * up1 + up2;
      S e0 = 1e-6 + (13.0 / 12.0 * (a0 * a0) + 1.0 / 4.0 * (b0 * b0));
      S e1 = 1e-6 + (13.0 / 12.0 * (a1 * a1) + 1.0 / 4.0 * (b1 * b1));
      S e2 = 1e-6 + (13.0 / 12.0 * (a2 * a2) + 1.0 / 4.0 * (b2 * b2));
      S s0 = e0 * e0, s1 = e1 * e1, s2 = e2 * e2;
      S q0 = -1.0 / 6.0 * um2 + 5.0 / 6.0 * um1 + 1.0 / 3.0 * u0;
      S q1 = 1.0 / 3.0 * um1 + 5.0 / 6.0 * u0 - 1.0 / 6.0 * up1;
      S q2 = 11.0 / 6.0 * u0 - 7.0 / 6.0 * up1 + 1.0 / 3.0 * up2;
      S w0b = 3.0 / 10.0 / s0, w1b = 6.0 / 10.0 / s1, w2b = 1.0 / 10.0 / s2;
      S sum = w0b + w1b + w2b;
      wL = w0b / sum * q0 + w1b / sum * q1 + w2b / sum * q2;
      q0 = 1.0 / 3.0 * um2 - 7.0 / 6.0 * um1 + 11.0 / 6.0 * u0;
      q1 = -1.0 / 6.0 * um1 + 5.0 / 6.0 * u0 + 1.0 / 3.0 * up1;
      q2 = 1.0 / 3.0 * u0 + 5.0 / 6.0 * up1 - 1.0 / 6.0 * up2;
      w0b = 1.0 / 10.0 / s0;
      w1b = 6.0 / 10.0 / s1;
      w2b = 3.0 / 10.0 / s2;
      sum = w0b + w1b + w2b;
      wR = w0b / sum * q0 + w1b / sum * q1 + w2b / sum * q2;
      break;
    }
  }
}

// ---------------------------------------------------------------- explicit fluxes
// The fast forms (kFast) take 1 / rho once where the reference divides by rho per term.
template <class S>
__device__ __forceinline__ void f_conv_fast(const S* c, int dir, S ir, S* f) {
  const S vx = c[1] * ir, vy = c[2] * ir, vz = c[3] * ir;
  const S k = 0.5 * c[0] * fma(vx, vx, fma(vy, vy, vz * vz));
  const S vn = dir == 0 ? vx : vy;
  const S mn = c[0] * vn;
  f[0] = mn;
  f[1] = mn * vx;
  f[2] = mn * vy;
  f[3] = mn * vz;
  f[4] = k * vn;
}
template <class S>
__device__ __forceinline__ void magflux_p_fast(const S* Q, int dir, S ir, S* f) {
  const S B2 = fma(Q[5], Q[5], fma(Q[6], Q[6], Q[7] * Q[7]));
  const S vB = fma(Q[1], Q[5], fma(Q[2], Q[6], Q[3] * Q[7])) * ir;
  const S Bn = dir == 0 ? Q[5] : Q[6];
  f[0] = 0;
  f[1] = dir == 0 ? fma(B2, S(0.5), -Q[5] * Q[5]) : -Q[5] * Q[6];
  f[2] = dir == 0 ? -Q[5] * Q[6] : fma(B2, S(0.5), -Q[6] * Q[6]);
  f[3] = -Bn * Q[7];
  f[4] = fma(Q[1 + dir] * ir, B2, -Bn * vB);
}
// convective flux along dir (0 = x, 1 = y), state.cpp:27-44 / 86-106
template <class S>
__device__ __forceinline__ void f_conv(const S* c, int dir, S* f) {
  S rho = c[0], vx = c[1] / c[0], vy = c[2] / c[0], vz = c[3] / c[0];
  S k = calkinetic(c);
  S vn = dir == 0 ? vx : vy;
  f[0] = rho * vn;
  f[1] = rho * vx * vn;
  f[2] = rho * vy * vn;
  f[3] = rho * vz * vn;
  f[4] = k * vn;
}
// magnetic flux of the pressure formula, state.cpp:298-322
template <class S>
__device__ __forceinline__ void magflux_p(const S* Q, int dir, S* f) {
  S B2 = Q[5] * Q[5] + Q[6] * Q[6] + Q[7] * Q[7];
  S vB = (Q[1] * Q[5] + Q[2] * Q[6] + Q[3] * Q[7]) / Q[0];
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
// magnetic flux of the energy formula, MagneticFlux_x/y (state.cpp:272-296)
template <class S>
__device__ __forceinline__ void magflux_e(const DevParams& P, const S* Q, int dir, S* f) {
  S B2 = Q[5] * Q[5] + Q[6] * Q[6] + Q[7] * Q[7];
  S vB = (Q[1] * Q[5] + Q[2] * Q[6] + Q[3] * Q[7]) / Q[0];
  f[0] = 0;
  if (dir == 0) {
    f[1] = (2 - P.gamma) * B2 * 0.5 - Q[5] * Q[5];
    f[2] = -Q[5] * Q[6];
    f[3] = -Q[5] * Q[7];
    f[4] = Q[1] / Q[0] * B2 * 0.5 - Q[5] * vB;
  } else {
    f[1] = -Q[5] * Q[6];
    f[2] = (2 - P.gamma) * B2 * 0.5 - Q[6] * Q[6];
    f[3] = -Q[6] * Q[7];
    f[4] = Q[2] / Q[0] * B2 * 0.5 - Q[6] * vB;
  }
}
// the non-zero component (1 + dir) of f/g_KineticEnergyFlux (state.cpp:325-345)
template <class S>
__device__ __forceinline__ S keflux(const DevParams& P, const S* Q) {
  return -(P.gamma - 1) * 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) / Q[0];
}
// total enthalpy (E + p) / rho, caltotalenthalpy (timestep.cpp:232-237)
template <class S>
__device__ __forceinline__ S caltotalenthalpy(const DevParams& P, const S* c) {
  S pri[8];
  con2pri(P, pri, c);
  return (c[4] + pri[4]) / pri[0];
}
// Rusanov face flux of RusanovC_x/y (flux.cpp:329-406), Pressure_flux_x/y (flux.cpp:202-287)
// or Energy_flux_x/y (flux.cpp:78-200): kForm 0, 1, 2
template <int kForm, bool kFast = false, class S>
__device__ __forceinline__ void face_flux(const DevParams& P, const S* QL, const S* QR, int dir, S a_max, S* F) {
  S fL[5], fR[5];
  if constexpr (kFast && kForm != 2) {
    const S irL = 1 / QL[0], irR = 1 / QR[0];
    f_conv_fast(QL, dir, irL, fL);
    f_conv_fast(QR, dir, irR, fR);
    if (kForm == 1) {
      S fb[5];
      magflux_p_fast(QL, dir, irL, fb);
#pragma unroll
      for (int k = 0; k < 5; ++k) fL[k] = fL[k] + fb[k];
      magflux_p_fast(QR, dir, irR, fb);
#pragma unroll
      for (int k = 0; k < 5; ++k) fR[k] = fR[k] + fb[k];
    } else if (P.formula == IMEX_EnergyFormula) {
      fL[4] = 0;
      fR[4] = 0;
    }
    const S s = P.GLF ? a_max : fmax(fabs(QL[1 + dir] * irL), fabs(QR[1 + dir] * irR));
    const S hs = 0.5 * s;
#pragma unroll
    for (int k = 0; k < 5; ++k) F[k] = fma(S(0.5), fL[k] + fR[k], -hs * (QR[k] - QL[k]));
    return;
  }
  f_conv(QL, dir, fL);
  f_conv(QR, dir, fR);
  if (kForm == 2) {  // convective (energy zeroed) + magnetic + kinetic-energy fluxes
    fL[4] = 0;
    fR[4] = 0;
    S fb[5];
    const S kl = keflux(P, QL), kr = keflux(P, QR);
    magflux_e(P, QL, dir, fb);
#pragma unroll
    for (int k = 0; k < 5; ++k) fL[k] = fL[k] + fb[k] + (k == 1 + dir ? kl : S(0.0));
    magflux_e(P, QR, dir, fb);
#pragma unroll
    for (int k = 0; k < 5; ++k) fR[k] = fR[k] + fb[k] + (k == 1 + dir ? kr : S(0.0));
  } else if (kForm == 1) {
    S fb[5];
    magflux_p(QL, dir, fb);
#pragma unroll
    for (int k = 0; k < 5; ++k) fL[k] = fL[k] + fb[k];
    magflux_p(QR, dir, fb);
#pragma unroll
    for (int k = 0; k < 5; ++k) fR[k] = fR[k] + fb[k];
  } else if (P.formula == IMEX_EnergyFormula) {
    fL[4] = 0;
    fR[4] = 0;
  }
  S s = P.GLF ? a_max : fmax(fabs(QL[1 + dir] / QL[0]), fabs(QR[1 + dir] / QR[0]));
#pragma unroll
  for (int k = 0; k < 5; ++k) F[k] = 0.5 * (fL[k] + fR[k]) - 0.5 * s * (QR[k] - QL[k]);
}

}  // namespace imex
