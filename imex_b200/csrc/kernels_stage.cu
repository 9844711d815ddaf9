// Explicit parts of one IMEX stage: step prologue (global wave-speed maxima
// and dt), stage combination, reconstruction, the two explicit flux updates,
// constrained transport, stage derivative, and diagnostics.
//
// Every kernel here is a memory-bound stencil over interior-only SoA planes
// with periodic or clamped neighbour indices (no ghost cells): one thread per cell, loads
// through the read-only path so the stencil neighbours hit L1.
#include <cstdio>
#include <cstring>

#include "cells.cuh"
#include "launch.cuh"

namespace imex {

namespace {

constexpr int kThreads = 256;

inline int blocks_for(long long n) { return (int)((n + kThreads - 1) / kThreads); }

// ---------------------------------------------------------------- reductions
template <typename T, typename F>
__device__ inline T warp_reduce(T v, F f) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = f(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
struct FMax {
  __device__ double operator()(double a, double b) const { return fmax(a, b); }
};
struct FMin {
  __device__ double operator()(double a, double b) const { return fmin(a, b); }
};
struct FSum {
  __device__ double operator()(double a, double b) const { return a + b; }
};
// block-wide reduction of K values; result valid in thread 0
template <int K, typename F>
__device__ inline void block_reduce(double (&v)[K], F f, double identity) {
  __shared__ double sh[K][kThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double r = warp_reduce(v[k], f);
    if (lane == 0) sh[k][wid] = r;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double r = lane < (int)(blockDim.x >> 5) ? sh[k][lane] : identity;
      v[k] = warp_reduce(r, f);
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------- step prologue
// calch / calca / caldt maxima / MagneticEigenvalues over the primitive state,
// timestep.cpp:5-148,254-273.  Max is exact, so block order does not matter.
constexpr int kStepVals = 11;
template <bool kFast>
struct k_step_reduce {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const double* __restrict__ prim, double* __restrict__ partial) {
    double v[kStepVals];
    v[0] = v[1] = v[2] = v[3] = v[4] = v[5] = 1e-8;  // ch_x ch_y ch cA_x cA_y cA
    v[6] = v[7] = v[8] = v[9] = v[10] = 0.0;         // |vx| |vy| |v| bmax_x bmax_y
    const long long N = P.N;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N; n += (long long)gridDim.x * blockDim.x) {
      double p[8];
      load_cell<8>(prim, N, n, p);
      double B2 = p[5] * p[5] + p[6] * p[6] + p[7] * p[7];
      double B = sqrt(B2);
      double vv = sqrt(p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
      if constexpr (kFast) {
        // one 1/rho and one 1/sqrt(rho) for the cell, the shared sound and Alfven terms of
        // the three fast speeds formed once (the exact form divides in every term)
        const double ir = 1.0 / p[0], isr = sqrt(ir);
        const double a2 = P.eos_type == IMEX_IDEAL_GAS ? P.gamma * p[4] * ir : eos_a2(P, p[0], p[4]);
        const double t = a2 + B2 * ir, tt = t * t, a4 = 4.0 * a2 * ir;
        auto cf_of = [&](double Bn) {
          double disc = tt - a4 * Bn * Bn;
          if (disc < 0) disc = 0;
          return sqrt(0.5 * (t + sqrt(disc)));
        };
        v[0] = fmax(v[0], p[1] + cf_of(p[5]));
        v[1] = fmax(v[1], p[2] + cf_of(p[6]));
        v[2] = fmax(v[2], vv + cf_of(B));
        v[3] = fmax(v[3], p[5] * isr);
        v[4] = fmax(v[4], p[6] * isr);
        v[5] = fmax(v[5], B * isr);
        v[6] = fmax(v[6], fabs(p[1]));
        v[7] = fmax(v[7], fabs(p[2]));
        v[8] = fmax(v[8], vv);
        const double b4 = 4 * B2 * ir;
        v[9] = fmax(v[9], 0.5 * (fabs(p[1]) + sqrt(p[1] * p[1] + b4)));
        v[10] = fmax(v[10], 0.5 * (fabs(p[2]) + sqrt(p[2] * p[2] + b4)));
        continue;
      }
      double cfx = eos_fast(P, p[0], p[4], p[5], B2);
      double cfy = eos_fast(P, p[0], p[4], p[6], B2);
      double cf = eos_fast(P, p[0], p[4], B, B2);
      v[0] = fmax(v[0], p[1] + cfx);
      v[1] = fmax(v[1], p[2] + cfy);
      v[2] = fmax(v[2], vv + cf);
      v[3] = fmax(v[3], p[5] / sqrt(p[0]));
      v[4] = fmax(v[4], p[6] / sqrt(p[0]));
      v[5] = fmax(v[5], B / sqrt(p[0]));
      v[6] = fmax(v[6], fabs(p[1]));
      v[7] = fmax(v[7], fabs(p[2]));
      v[8] = fmax(v[8], vv);
      v[9] = fmax(v[9], 0.5 * (fabs(p[1]) + sqrt(p[1] * p[1] + 4 * B2 / p[0])));
      v[10] = fmax(v[10], 0.5 * (fabs(p[2]) + sqrt(p[2] * p[2] + 4 * B2 / p[0])));
    }
    block_reduce(v, FMax(), -INFINITY);
    if (threadIdx.x == 0)
      for (int k = 0; k < kStepVals; ++k) partial[blockIdx.x * kStepVals + k] = v[k];
  }
};

// caldt (timestep.cpp:5-67) + main.cpp:341-353 on one thread
struct k_step_finalize {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const double* __restrict__ partial, int nblk, DevScalars* sc) {
    double v[kStepVals];
    for (int k = 0; k < kStepVals; ++k) v[k] = -INFINITY;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
      for (int k = 0; k < kStepVals; ++k) v[k] = fmax(v[k], partial[b * kStepVals + k]);
    block_reduce(v, FMax(), -INFINITY);
    if (threadIdx.x != 0) return;
    sc->timestep += 1;
    const int ts = sc->timestep;
    sc->ch_x = v[0];
    sc->ch_y = v[1];
    sc->ch = v[2];
    sc->cA_x = v[3];
    sc->cA_y = v[4];
    sc->cA = v[5];
    sc->vx_max = v[6];
    sc->vy_max = v[7];
    sc->v_max = v[8];
    const int full_step = 1;
    double a_max;
    if (P.caltimestep == IMEX_Fullydt) a_max = sc->ch;
    else if (P.caltimestep == IMEX_Alfvendt) a_max = (ts < full_step + 1) ? sc->ch : sc->cA;
    else a_max = (ts < full_step + 1) ? sc->ch : sc->v_max;
    double dt = P.CFL * 1 / (2 * a_max / fmin(P.dx, P.dy));
    if (ts > 1 && sc->prev_dt > 0.0) dt = fmin(dt, 2.0 * sc->prev_dt);
    sc->prev_dt = dt;
    if (ts > full_step) a_max = sc->v_max;
    sc->a_max = a_max;
    dt = fmin(dt, P.time_stop - sc->t);
    if (P.fixed_dt > 0.0) dt = fmin(P.fixed_dt, P.time_stop - sc->t);
    sc->dt = dt;
    sc->B_max_x = v[9];
    sc->B_max_y = v[10];
    sc->t = sc->t + dt;
  }
};

// cons = pri2con(prim); cons_n = cons  (main.cpp:356-358)
struct k_cons_from_prim {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const double* __restrict__ prim, double* __restrict__ cons,
                                   double* __restrict__ cons_n) {
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= P.N) return;
    double p[8], c[8];
    load_cell<8>(prim, P.N, n, p);
    pri2con(P, c, p);
  #pragma unroll
    for (int k = 0; k < 8; ++k) {
      cons[k * P.N + n] = c[k];
      if (cons_n) cons_n[k * P.N + n] = c[k];
    }
  }
};
__global__ void k_prim_from_cons(DevParams P, const double* __restrict__ cons, double* __restrict__ prim) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= P.N) return;
  double p[8], c[8];
  load_cell<8>(cons, P.N, n, c);
  con2pri(P, p, c);
#pragma unroll
  for (int k = 0; k < 8; ++k) prim[k * P.N + n] = p[k];
}

// ---------------------------------------------------------------- stage combination
struct Tableau {
  double ae[kMaxRK], ai[kMaxRK], aii;
};
// Qe, Qs, face and A stage states (main.cpp:368-414), plus the pressure and
// enthalpy of Qe that the implicit sub-systems freeze for the stage.
// R = rks: the stage count is a template parameter so that every load of a thread is
// issued before the first is used.  kG: the A form also takes the global A-viscosity
// maxima of prim(Qs) (implicit_operators.cpp:364-374, the k_gmax expression) from the Qs
// it has just formed, one fmax pair per CTA into partial[2 * block], which saves the
// separate pass over Qs.
template <int R, bool kG>
struct k_stage_combine {
  IMEX_BOUNDS(kThreads, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, Tableau T, DevScalars* sc, const double* __restrict__ cons_n,
                                  const double* __restrict__ Hs, const double* __restrict__ bx_n,
                                  const double* __restrict__ by_n, const double* __restrict__ HsB,
                                  const double* __restrict__ A_snap, const double* __restrict__ HsA,
                                  double* __restrict__ Qe, double* __restrict__ Qs, double* __restrict__ bxQe,
                                  double* __restrict__ byQe, double* __restrict__ bxQs, double* __restrict__ byQs,
                                  double* __restrict__ A_s, double* __restrict__ A_e, double* __restrict__ A,
                                  double* __restrict__ pe, double* __restrict__ hQe,
                                  double* __restrict__ partial) {
    const long long N = P.N;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const double dt = sc->dt;
    if (n == 0) {
      sc->adt = T.aii * dt;
      sc->h = T.aii * dt;
    }
    double g0 = 0.0, g1 = 0.0;
    if (n < N) {
    constexpr int RR = R > 0 ? R : 1;
    double u[8], h[RR][8], a[3], ha[RR][3], fx = bx_n[n], fy = by_n[n], hb[RR][2];
  #pragma unroll
    for (int k = 0; k < 8; ++k) u[k] = cons_n[k * N + n];
  #pragma unroll
    for (int k = 0; k < 3; ++k) a[k] = A_snap[k * N + n];
  #pragma unroll
    for (int r = 0; r < R; ++r) {
  #pragma unroll
      for (int k = 0; k < 8; ++k) h[r][k] = Hs[((long long)r * 8 + k) * N + n];
  #pragma unroll
      for (int k = 0; k < 3; ++k) ha[r][k] = HsA[((long long)r * 3 + k) * N + n];
      hb[r][0] = HsB[((long long)r * 2 + 0) * N + n];
      hb[r][1] = HsB[((long long)r * 2 + 1) * N + n];
    }
    double qe[8], qs[8];
  #pragma unroll
    for (int k = 0; k < 8; ++k) {
      double e = u[k], s = e;
  #pragma unroll
      for (int r = 0; r < R; ++r) {
        e = e + T.ae[r] * dt * h[r][k];
        s = s + T.ai[r] * dt * h[r][k];
      }
      qe[k] = e;
      qs[k] = s;
      Qe[k * N + n] = e;
      Qs[k * N + n] = s;
    }
  #pragma unroll
    for (int k = 0; k < 3; ++k) {
      double e = a[k], s = e;
  #pragma unroll
      for (int r = 0; r < R; ++r) {
        e += T.ae[r] * dt * ha[r][k];
        s += T.ai[r] * dt * ha[r][k];
      }
      A_e[k * N + n] = e;
      A_s[k * N + n] = s;
      A[k * N + n] = s;
    }
    double fxe = fx, fxs = fxe, fye = fy, fys = fye;
  #pragma unroll
    for (int r = 0; r < R; ++r) {
      fxe += T.ae[r] * dt * hb[r][0];
      fye += T.ae[r] * dt * hb[r][1];
      fxs += T.ai[r] * dt * hb[r][0];
      fys += T.ai[r] * dt * hb[r][1];
    }
    bxQe[n] = fxe;
    byQe[n] = fye;
    bxQs[n] = fxs;
    byQs[n] = fys;
    double e = calecon(qe);
    double p = eos_p(P, qe[0], e);
    pe[n] = p;
    hQe[n] = e + p / qe[0];
    if constexpr (kG) {
      const double vx = qs[1] / qs[0], vy = qs[2] / qs[0];
      const double Bsq = qs[5] * qs[5] + qs[6] * qs[6] + qs[7] * qs[7];
      g0 = fmax(g0, 0.5 * (fabs(vx) + sqrt(vx * vx + 4.0 * Bsq / qs[0])));
      g1 = fmax(g1, 0.5 * (fabs(vy) + sqrt(vy * vy + 4.0 * Bsq / qs[0])));
    }
    }
    if constexpr (kG) {
      __shared__ double sh[2][kThreads / 32];
      for (int o = 16; o > 0; o >>= 1) {
        g0 = fmax(g0, __shfl_xor_sync(0xffffffffu, g0, o));
        g1 = fmax(g1, __shfl_xor_sync(0xffffffffu, g1, o));
      }
      if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = g0;
        sh[1][threadIdx.x >> 5] = g1;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        for (int w = 1; w < kThreads / 32; ++w) {
          g0 = fmax(g0, sh[0][w]);
          g1 = fmax(g1, sh[1][w]);
        }
        partial[2 * blockIdx.x] = g0;
        partial[2 * blockIdx.x + 1] = g1;
      }
    }
  }
};

// ---------------------------------------------------------------- reconstruction
// TVDReconstruction (reconstruction.cpp:5-287) of Q into w = [xL | xR | yL | yR] x 8 planes,
// PrimState (the ConsState form is k_reconstruct_var below).
// nstore = number of conserved variables written (5 for the stage, 8 for the full buffer).
template <bool kOpen, bool kFast>
struct k_reconstruct_prim {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams Pin, const double* __restrict__ Q, double* __restrict__ w, int nstore) {
    const DevParams P = bc_params<kOpen>(Pin);
    const long long N = P.N;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    int i, j;
    cell_of(P, n, i, j);
    long long ix[5], iy[5];
  #pragma unroll
    for (int d = 0; d < 5; ++d) {
      ix[d] = cid(P, i + d - 2, j);
      iy[d] = cid(P, i, j + d - 2);
    }
    const bool vortex = P.recon == IMEX_Minmod && P.vortex_minmod;
    // PrimState: reconstruct primitive variables, convert each face state back (reconstruction.cpp:272-281)
    double px[5][8], py[5][8];
  #pragma unroll
    for (int d = 0; d < 5; ++d) {
      double c[8];
      load_cell<8>(Q, N, ix[d], c);
      con2pri(P, px[d], c);
      load_cell<8>(Q, N, iy[d], c);
      con2pri(P, py[d], c);
    }
    double wxl[8], wxr[8], wyl[8], wyr[8];
  #pragma unroll
    for (int k = 0; k < 8; ++k) {
      recon_1d<kFast>(P.recon, px[0][k], px[1][k], px[2][k], px[3][k], px[4][k], wxl[k], wxr[k], false);
      recon_1d<kFast>(P.recon, py[0][k], py[1][k], py[2][k], py[3][k], py[4][k], wyl[k], wyr[k], vortex);
    }
    double c[8];
    double* outs[4] = {wxl, wxr, wyl, wyr};
  #pragma unroll
    for (int q = 0; q < 4; ++q) {
      pri2con(P, c, outs[q]);
      for (int k = 0; k < nstore; ++k) w[(q * 8 + k) * N + n] = c[k];
    }
  }
};

// ConsState reconstructs every conserved variable on its own (reconstruction.cpp:5-266), so
// one thread per (cell, variable) pair: variable k = blockIdx.y.  The same recon_1d calls as a
// per-cell loop over the variables, with a small per-thread working set and 5-8x the threads.
template <bool kOpen, bool kFast>
struct k_reconstruct_var {
  IMEX_BOUNDS(kThreads, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams Pin, const double* __restrict__ Q,
                                                                 double* __restrict__ w) {
    const DevParams P = bc_params<kOpen>(Pin);
    const long long N = P.N;
    const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int k = blockIdx.y;
    int i, j;
    cell_of(P, n, i, j);
    const bool vortex = P.recon == IMEX_Minmod && P.vortex_minmod;
    const double* a = Q + k * N;
    double v[5], u[5];  // both stencils loaded before the divisions of the first reconstruction
  #pragma unroll
    for (int d = 0; d < 5; ++d) v[d] = __ldg(a + cid(P, i + d - 2, j));
  #pragma unroll
    for (int d = 0; d < 5; ++d) u[d] = __ldg(a + cid(P, i, j + d - 2));
    double xl, xr, yl, yr;
    if (kFast && P.recon == IMEX_WENO5) {
      weno5_fast_xy(v, u, xl, xr, yl, yr);
    } else {
      recon_1d<kFast>(P.recon, v[0], v[1], v[2], v[3], v[4], xl, xr, false);
      recon_1d<kFast>(P.recon, u[0], u[1], u[2], u[3], u[4], yl, yr, vortex);
    }
    w[(0 * 8 + k) * N + n] = xl;
    w[(1 * 8 + k) * N + n] = xr;
    w[(2 * 8 + k) * N + n] = yl;
    w[(3 * 8 + k) * N + n] = yr;
  }
};

// ---------------------------------------------------------------- flux updates
// RusanovC_Update (flux.cpp:409-455) or Pressure_flux_Update (flux.cpp:290-326) with the
// B slots of the face states taken from cell B of u_con (main.cpp:447-467).
// Each face flux of a 32 x 8 tile is evaluated once (the cells of the tile share their
// faces: 552 face fluxes for 256 cells, against 4 per cell when every cell evaluates its
// own), kept in shared memory, then each cell is updated with the reference's expression:
// fp / fm are the fluxes of the faces at i +- 1/2, gp / gm those at j +- 1/2.
constexpr int FTX = 32, FTY = 8, FNT = FTX * FTY;
template <int kForm, bool kFast>
__device__ __forceinline__ void flux_tile(IMEX_BLK, const DevParams& P, const DevScalars* __restrict__ sc,
                                          const double* __restrict__ w, const double* __restrict__ Qs,
                                          double* __restrict__ ucon) {
  __shared__ double fx[5][FTY][FTX + 1];  // fx[.][ly][fi]: face between cells x0 + fi - 1 and x0 + fi
  __shared__ double fy[5][FTY + 1][FTX];  // fy[.][fj][lx]: face between cells y0 + fj - 1 and y0 + fj
  const long long N = P.N;
  const double h = sc->h, a_max = sc->a_max;
  const int x0 = blockIdx.x * FTX, y0 = blockIdx.y * FTY;
  const int ncol = P.nx - x0 < FTX ? P.nx - x0 : FTX, nrow = P.ny - y0 < FTY ? P.ny - y0 : FTY;
  const double* wxL = w;
  const double* wxR = w + 8 * N;
  const double* wyL = w + 16 * N;
  const double* wyR = w + 24 * N;
  auto state = [&](const double* wq, long long m, double* Q) {
#pragma unroll
    for (int k = 0; k < 5; ++k) Q[k] = __ldg(wq + k * N + m);
    if (kForm != 0) {
#pragma unroll
      for (int k = 5; k < 8; ++k) Q[k] = __ldg(ucon + k * N + m);
    } else {
      Q[5] = Q[6] = Q[7] = 0.0;
    }
  };
  constexpr int NXF = (FTX + 1) * FTY, NYF = FTX * (FTY + 1);
  for (int f = threadIdx.x; f < NXF + NYF; f += FNT) {
    double QL[8], QR[8], F[5];
    if (f < NXF) {
      const int fi = f % (FTX + 1), ly = f / (FTX + 1);
      if (fi > ncol || ly >= nrow) continue;
      const int j = y0 + ly;
      state(wxR, cid(P, x0 + fi - 1, j), QL);
      state(wxL, cid(P, x0 + fi, j), QR);
      face_flux<kForm, kFast>(P, QL, QR, 0, a_max, F);
#pragma unroll
      for (int k = 0; k < 5; ++k) fx[k][ly][fi] = F[k];
    } else {
      const int g = f - NXF, lx = g % FTX, fj = g / FTX;
      if (lx >= ncol || fj > nrow) continue;
      const int i = x0 + lx;
      state(wyR, cid(P, i, y0 + fj - 1), QL);
      state(wyL, cid(P, i, y0 + fj), QR);
      face_flux<kForm, kFast>(P, QL, QR, 1, a_max, F);
#pragma unroll
      for (int k = 0; k < 5; ++k) fy[k][fj][lx] = F[k];
    }
  }
  __syncthreads();
  const int lx = threadIdx.x % FTX, ly = threadIdx.x / FTX;
  if (lx >= ncol || ly >= nrow) return;
  const long long n = (long long)(y0 + ly) * P.nx + (x0 + lx);
#pragma unroll
  for (int k = 0; k < 5; ++k)
    ucon[k * N + n] = Qs[k * N + n] - h / P.dx * (fx[k][ly][lx + 1] - fx[k][ly][lx]) -
                      h / P.dy * (fy[k][ly + 1][lx] - fy[k][ly][lx]);
}
// The register budgets were measured: the convective form runs fastest as the compiler
// chooses, the pressure and energy forms at three CTAs per SM.
template <bool kOpen, bool kFast>
struct k_flux_conv {
  // the fast instance fits 64 registers (four CTAs per SM); the bound keeps it there
  static constexpr int kNT = FNT, kMinB = kFast ? 4 : 0;
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams Pin, const DevScalars* __restrict__ sc,
                                                     const double* __restrict__ w, const double* __restrict__ Qs,
                                                     double* __restrict__ ucon) {
    const DevParams P = bc_params<kOpen>(Pin);
    flux_tile<0, kFast>(blockIdx, gridDim, P, sc, w, Qs, ucon);
  }
};
template <int kForm, bool kOpen, bool kFast>
struct k_flux_mag {
  IMEX_BOUNDS(FNT, 3)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams Pin, const DevScalars* __restrict__ sc,
                                                       const double* __restrict__ w, const double* __restrict__ Qs,
                                                       double* __restrict__ ucon) {
    const DevParams P = bc_params<kOpen>(Pin);
    flux_tile<kForm, kFast>(blockIdx, gridDim, P, sc, w, Qs, ucon);
  }
};
template <bool kOpen, bool kFast>
struct k_flux_pres {
  IMEX_BOUNDS(FNT, 3)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams Pin, const DevScalars* __restrict__ sc,
                                                        const double* __restrict__ w, const double* __restrict__ Qs,
                                                        double* __restrict__ ucon) {
    const DevParams P = bc_params<kOpen>(Pin);
    flux_tile<1, kFast>(blockIdx, gridDim, P, sc, w, Qs, ucon);
  }
};

// ---------------------------------------------------------------- constrained transport
// corner EMF (ci + 1/2, cj + 1/2) for ci, cj >= -1 (ct_corner_at): Ez_bar on the corner
// index as bound_cond_array leaves it (clamped to 0 on x_0 / y_0 of a transmissive
// direction, the periodic image otherwise), the correction terms on the corner itself
template <class Ld>
__device__ __forceinline__ double corner_emf(const DevParams& P, double sx, double sy, int ci, int cj, Ld& ld) {
  long long nb[9], bnb[9];
  neighbours(P, ci, cj, nb);
  const int bi = ci < 0 ? (P.xclamp ? 0 : P.nx + ci) : ci, bj = cj < 0 ? (P.yclamp ? 0 : P.ny + cj) : cj;
  neighbours(P, bi, bj, bnb);
  double out[1];
  ct_corner_at<double>(P, sx, sy, nb, bnb, ld, out);
  return out[0];
}
// Corner EMF of u_con and the collected face fluxes (ct_corner_cell); on a transmissive
// direction the first column / row of threads also writes the boundary corners (-1/2).
struct k_ct_corner {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const double* __restrict__ fx, double sx, const double* __restrict__ fy,
                              double sy, const double* __restrict__ ucon, double* __restrict__ Epp, BoundaryLines L) {
    const long long N = P.N;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    int i, j;
    cell_of(P, n, i, j);
    long long nb[9];
    neighbours(P, i, j, nb);
    const double* arr[3] = {fx, fy, ucon};
    auto ld = [&](int a, int k, long long m) { return __ldg(arr[a] + k * N + m); };
    double out[1];
    ct_corner_cell<double>(P, sx, sy, nb, ld, out);
    Epp[n] = out[0];
    if (P.xclamp && i == 0) {
      L.ex[j + 1] = corner_emf(P, sx, sy, -1, j, ld);
      if (j == 0) L.ex[0] = corner_emf(P, sx, sy, -1, -1, ld);
    }
    if (P.yclamp && j == 0) {
      L.ey[i + 1] = corner_emf(P, sx, sy, i, -1, ld);
      if (i == 0) L.ey[0] = corner_emf(P, sx, sy, -1, -1, ld);
    }
  }
};
// corner (ci + 1/2, cj + 1/2), ci, cj >= -1, from the corner plane and the boundary lines
__device__ __forceinline__ double corner_read(const DevParams& P, const double* __restrict__ Epp,
                                              const BoundaryLines& L, int ci, int cj) {
  if (ci < 0 && P.xclamp) return L.ex[cj + 1];
  if (cj < 0 && P.yclamp) return L.ey[cix(P, ci) + 1];
  return __ldg(Epp + cid(P, ci, cj));
}
// Face update from the corner EMF and cell B = face average
// (ct_flux.cpp:174-189, constrained_transport.cpp:128-141).  The neighbour faces
// are recomputed with the same arithmetic rather than re-read.
// On a transmissive direction the faces left of / below the first column / row are the
// boundary faces (their own lines, corner EMFs from the boundary corners), which the
// first column / row of threads also stores.
struct k_ct_faces {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const DevScalars* __restrict__ sc, const double* __restrict__ Epp,
                             const double* __restrict__ bxQs, const double* __restrict__ byQs, double* __restrict__ bx,
                             double* __restrict__ by, double* __restrict__ ucon, BoundaryLines L) {
    const long long N = P.N;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    int i, j;
    cell_of(P, n, i, j);
    const double h = sc->h;
    const bool xb = P.xclamp && i == 0, yb = P.yclamp && j == 0;
    double e00 = __ldg(Epp + n), em0 = corner_read(P, Epp, L, i - 1, j), e0m = corner_read(P, Epp, L, i, j - 1);
    double emm = corner_read(P, Epp, L, i - 1, j - 1);
    double fx = __ldg(bxQs + n) - h / P.dy * (e00 - e0m);
    double fy = __ldg(byQs + n) + h / P.dx * (e00 - em0);
    double fxm = (xb ? L.bxQs[j] : __ldg(bxQs + cid(P, i - 1, j))) - h / P.dy * (em0 - emm);
    double fym = (yb ? L.byQs[i] : __ldg(byQs + cid(P, i, j - 1))) + h / P.dx * (e0m - emm);
    bx[n] = fx;
    by[n] = fy;
    if (xb) L.bx[j] = fxm;
    if (yb) L.by[i] = fym;
    ucon[5 * N + n] = 0.5 * (fxm + fx);
    ucon[6 * N + n] = 0.5 * (fym + fy);
  }
};
// Stage combination (main.cpp:397-407) and stage derivative (main.cpp:550-551) of the
// boundary-face lines of the transmissive directions; thread q handles row q of the x_0
// line and column q of the y_0 line.
struct k_bline_combine {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, Tableau T, int rks, const DevScalars* __restrict__ sc, BoundaryLines L) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const double dt = sc->dt;
    if (P.xclamp && q < P.ny) {
      double fe = L.bx_n[q], fs = fe;
      for (int r = 0; r < rks; ++r) {
        const double h0 = L.hsbx[(long long)r * P.ny + q];
        fe += T.ae[r] * dt * h0;
        fs += T.ai[r] * dt * h0;
      }
      L.bxQe[q] = fe;
      L.bxQs[q] = fs;
    }
    if (P.yclamp && q < P.nx) {
      double fe = L.by_n[q], fs = fe;
      for (int r = 0; r < rks; ++r) {
        const double h1 = L.hsby[(long long)r * P.nx + q];
        fe += T.ae[r] * dt * h1;
        fs += T.ai[r] * dt * h1;
      }
      L.byQe[q] = fe;
      L.byQs[q] = fs;
    }
  }
};
struct k_bline_derivative {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, int rks, const DevScalars* __restrict__ sc, BoundaryLines L) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const double adt = sc->adt;
    if (P.xclamp && q < P.ny) L.hsbx[(long long)rks * P.ny + q] = (L.bx[q] - L.bxQs[q]) / adt;
    if (P.yclamp && q < P.nx) L.hsby[(long long)rks * P.nx + q] = (L.by[q] - L.byQs[q]) / adt;
  }
};
// Unstaggered_CT_Consistent A_z update (constrained_transport.cpp:523-529)
struct k_ct_unstag_A {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const DevScalars* __restrict__ sc, const double* __restrict__ Epp,
                                const double* __restrict__ A_s, double* __restrict__ A, BoundaryLines L) {
    const long long N = P.N;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    int i, j;
    cell_of(P, n, i, j);
    double Ec = 0.25 * (__ldg(Epp + n) + corner_read(P, Epp, L, i - 1, j) + corner_read(P, Epp, L, i, j - 1) +
                        corner_read(P, Epp, L, i - 1, j - 1));
    A[2 * N + n] = A_s[2 * N + n] - sc->h * Ec;
  }
};
// Unstaggered_CT upwind A_z advection (constrained_transport.cpp:436-488); A_s is read with
// the ghosts of bound_cond_A (constrained_transport.cpp:438), u_con with those of bound_cond_u
__device__ __forceinline__ double vanleer_lim(double a, double b) {
  if (a * b <= 0.0) return 0.0;
  return 2.0 * a * b / (a + b);
}
struct k_ct_unstag_legacy_A {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const DevScalars* __restrict__ sc, const double* __restrict__ u,
                                       const double* __restrict__ A_s, double* __restrict__ A) {
    const long long N = P.N;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    int i, j;
    cell_of(P, n, i, j);
    const double h = sc->h, dx = P.dx, dy = P.dy;
    const double* As = A_s + 2 * N;
    auto vxc = [&](long long m) { return __ldg(u + N + m) / __ldg(u + m); };
    auto vyc = [&](long long m) { return __ldg(u + 2 * N + m) / __ldg(u + m); };
    const long long c = n, xm = cid(P, i - 1, j), xp = cid(P, i + 1, j), ym = cid(P, i, j - 1), yp = cid(P, i, j + 1);
    const double a00 = As[c], axm = a_ghost(P, As, i - 1, j), axp = a_ghost(P, As, i + 1, j);
    const double axmm = a_ghost(P, As, i - 2, j), axpp = a_ghost(P, As, i + 2, j);
    const double aym = a_ghost(P, As, i, j - 1), ayp = a_ghost(P, As, i, j + 1);
    const double aymm = a_ghost(P, As, i, j - 2), aypp = a_ghost(P, As, i, j + 2);
    double uL = 0.5 * (vxc(xm) + vxc(c)), uR = 0.5 * (vxc(c) + vxc(xp));
    double dAL = a00 - axm, dAR = axp - a00, dALL = axm - axmm, dARR = axpp - axp;
    double fluct_x = fmax(uL, 0.0) * dAL + fmin(uR, 0.0) * dAR;
    double corrL = 0.5 * fabs(uL) * (1.0 - fabs(uL) * h / dx) * vanleer_lim(dAL, (uL >= 0.0 ? dALL : dAR));
    double corrR = 0.5 * fabs(uR) * (1.0 - fabs(uR) * h / dx) * vanleer_lim(dAR, (uR >= 0.0 ? dAL : dARR));
    double dAdt_x = fluct_x / dx + (corrR - corrL) / dx;
    double vL = 0.5 * (vyc(ym) + vyc(c)), vR = 0.5 * (vyc(c) + vyc(yp));
    double dAB = a00 - aym, dAT = ayp - a00, dABB = aym - aymm, dATT = aypp - ayp;
    double fluct_y = fmax(vL, 0.0) * dAB + fmin(vR, 0.0) * dAT;
    double corrB = 0.5 * fabs(vL) * (1.0 - fabs(vL) * h / dy) * vanleer_lim(dAB, (vL >= 0.0 ? dABB : dAT));
    double corrT = 0.5 * fabs(vR) * (1.0 - fabs(vR) * h / dy) * vanleer_lim(dAT, (vR >= 0.0 ? dAB : dATT));
    double dAdt_y = fluct_y / dy + (corrT - corrB) / dy;
    A[2 * N + n] = a00 - h * (dAdt_x + dAdt_y);
  }
};
// B = curl A_z for the unstaggered schemes (constrained_transport.cpp:533-538)
struct k_curl_Az {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const double* __restrict__ A, double* __restrict__ ucon) {
    const long long N = P.N;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    int i, j;
    cell_of(P, n, i, j);
    const double* Az = A + 2 * N;
    ucon[5 * N + n] = (a_ghost(P, Az, i, j + 1) - a_ghost(P, Az, i, j - 1)) / (2.0 * P.dy);
    ucon[6 * N + n] = -(a_ghost(P, Az, i + 1, j) - a_ghost(P, Az, i - 1, j)) / (2.0 * P.dx);
  }
};
// Face EMFs of the legacy Staggered_CT from the reconstruction of u_con
// (constrained_transport.cpp:73-97): Ez_p0 = -(f6_L + f6_R)/2, Ez_0p = (g5_L + g5_R)/2.
struct k_ct_legacy_faces {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const double* __restrict__ w, double* __restrict__ ep0,
                                    double* __restrict__ e0p) {
    const long long N = P.N;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    int i, j;
    cell_of(P, n, i, j);
    const double *wxL = w, *wxR = w + 8 * N, *wyL = w + 16 * N, *wyR = w + 24 * N;
    auto f6 = [&](const double* q, long long m) {
      double r = __ldg(q + m);
      return __ldg(q + 6 * N + m) * (__ldg(q + N + m) / r) - (__ldg(q + 2 * N + m) / r) * __ldg(q + 5 * N + m);
    };
    auto g5 = [&](const double* q, long long m) {
      double r = __ldg(q + m);
      return __ldg(q + 5 * N + m) * (__ldg(q + 2 * N + m) / r) - (__ldg(q + N + m) / r) * __ldg(q + 6 * N + m);
    };
    ep0[n] = -(0.5 * (f6(wxR, n) + f6(wxL, cid(P, i + 1, j))));
    e0p[n] = (0.5 * (g5(wyR, n) + g5(wyL, cid(P, i, j + 1))));
  }
};

// ---------------------------------------------------------------- CT EMF diagnostics
// Diagnose_CT_EMF (constrained_transport.cpp:183-222), printed by the reference's driver after
// every step (main.cpp:594).  The face EMFs of the reconstructed u_con split into their central
// average (C: -(f6_L + f6_R)/2 and (g5_L + g5_R)/2) and their Rusanov dissipation (R), plus the
// cell EMF Ez~ (T); CT_CornerAssemble turns each into corner EMFs with the other inputs zero.
__global__ void k_ct_diag_faces(DevParams P, const double* __restrict__ w, double* __restrict__ cp0,
                                double* __restrict__ c0p, double* __restrict__ rp0, double* __restrict__ r0p) {
  const long long N = P.N;
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  int i, j;
    cell_of(P, n, i, j);
  const double *wxL = w, *wxR = w + 8 * N, *wyL = w + 16 * N, *wyR = w + 24 * N;
  auto f6 = [&](const double* q, long long m) {  // f_full_con[6], state.cpp:152-175
    double r = __ldg(q + m);
    return __ldg(q + 6 * N + m) * (__ldg(q + N + m) / r) - (__ldg(q + 2 * N + m) / r) * __ldg(q + 5 * N + m);
  };
  auto g5 = [&](const double* q, long long m) {  // g_full_con[5], state.cpp:179-200
    double r = __ldg(q + m);
    return __ldg(q + 5 * N + m) * (__ldg(q + 2 * N + m) / r) - (__ldg(q + N + m) / r) * __ldg(q + 6 * N + m);
  };
  auto q = [&](const double* a, int k, long long m) { return __ldg(a + k * N + m); };
  const long long xp = cid(P, i + 1, j), yp = cid(P, i, j + 1);
  cp0[n] = -(0.5 * (f6(wxR, n) + f6(wxL, xp)));
  rp0[n] = 0.5 * fmax(fabs(q(wxR, 1, n) / q(wxR, 0, n)), fabs(q(wxL, 1, xp) / q(wxL, 0, xp))) *
           (q(wxL, 6, xp) - q(wxR, 6, n));
  c0p[n] = 0.5 * (g5(wyR, n) + g5(wyL, yp));
  r0p[n] = -0.5 * fmax(fabs(q(wyR, 2, n) / q(wyR, 0, n)), fabs(q(wyL, 2, yp) / q(wyL, 0, yp))) *
           (q(wyL, 5, yp) - q(wyR, 5, n));
}
// CT_EMF_Stats (constrained_transport.cpp:166-181) of C, R, T and their sum: per block the
// sums of dx dy Ez^2 and dx dy |dB/dt|^2 (slots 0-7) and the maxima of |Ez| and |dB/dt|
// (slots 8-15), where dB/dt = (-(E(i,j) - E(i,j-1))/dy, (E(i,j) - E(i-1,j))/dx) on the faces.
__global__ void k_ct_diag_stats(DevParams P, const double* __restrict__ cp0, const double* __restrict__ c0p,
                                const double* __restrict__ rp0, const double* __restrict__ r0p,
                                const double* __restrict__ ucon, double* __restrict__ partial) {
  const long long N = P.N;
  double sum[8] = {0, 0, 0, 0, 0, 0, 0, 0}, mx[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const double* fx[3] = {cp0, rp0, nullptr};
  const double* fy[3] = {c0p, r0p, nullptr};
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N; n += (long long)gridDim.x * blockDim.x) {
    int i, j;
    cell_of(P, n, i, j);
    double e[4][3];  // component (C, R, T, total) x corner ((i, j), (i, j-1), (i-1, j))
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      // C and R: their face EMFs and a zero cell EMF (rho 1, B 0); T: zero face EMFs and Ez~(u_con)
      auto ld = [&](int a, int k, long long m) -> double {
        if (a == CC_UCON) return c == 2 ? __ldg(ucon + k * N + m) : (k == 0 ? 1.0 : 0.0);
        if (c == 2) return 0.0;
        return __ldg((a == CC_FX ? fx[c] : fy[c]) + m);
      };
      e[c][0] = corner_emf(P, 1.0, 1.0, i, j, ld);
      e[c][1] = corner_emf(P, 1.0, 1.0, i, j - 1, ld);
      e[c][2] = corner_emf(P, 1.0, 1.0, i - 1, j, ld);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) e[3][k] = e[0][k] + e[1][k] + e[2][k];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double ez = e[c][0];
      sum[c] += P.dx * P.dy * ez * ez;
      mx[c] = fmax(mx[c], fabs(ez));
      const double dBx = -(e[c][0] - e[c][1]) / P.dy, dBy = (e[c][0] - e[c][2]) / P.dx;
      const double m2 = dBx * dBx + dBy * dBy;
      sum[4 + c] += P.dx * P.dy * m2;
      mx[4 + c] = fmax(mx[4 + c], sqrt(m2));
    }
  }
  block_reduce(sum, FSum(), 0.0);
  block_reduce(mx, FMax(), 0.0);
  if (threadIdx.x == 0)
    for (int k = 0; k < 8; ++k) {
      partial[blockIdx.x * 16 + k] = sum[k];
      partial[blockIdx.x * 16 + 8 + k] = mx[k];
    }
}

// ---------------------------------------------------------------- stage derivative
// Energy_Modify (main.cpp:528-534), Hs / HsA / HsB (main.cpp:539-555), u_pri (main.cpp:537).
struct k_stage_derivative {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, int rks, const DevScalars* __restrict__ sc, double* __restrict__ cons,
                                     const double* __restrict__ Qs, const double* __restrict__ A,
                                     const double* __restrict__ A_s, const double* __restrict__ bx,
                                     const double* __restrict__ bxQs, const double* __restrict__ by,
                                     const double* __restrict__ byQs, const double* __restrict__ Bsave,
                                     double* __restrict__ Hs, double* __restrict__ HsA, double* __restrict__ HsB,
                                     double* __restrict__ prim) {
    const long long N = P.N;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    const double adt = sc->adt;
    // every input first, so that the divisions below do not serialise the loads
    double c[8], qs[8], a[3], as[3], o[3];
    load_cell<8>(cons, N, n, c);
  #pragma unroll
    for (int k = 0; k < 8; ++k) qs[k] = Qs[k * N + n];
  #pragma unroll
    for (int k = 0; k < 3; ++k) {
      a[k] = A[k * N + n];
      as[k] = A_s[k * N + n];
    }
    const double fx = bx[n], fxs = bxQs[n], fy = by[n], fys = byQs[n];
    if (P.Energy_Modify) {
  #pragma unroll
      for (int k = 0; k < 3; ++k) o[k] = Bsave[k * N + n];
      c[4] = c[4] + ((c[5] * c[5] + c[6] * c[6] + c[7] * c[7]) - (o[0] * o[0] + o[1] * o[1] + o[2] * o[2])) / 2.0;
      cons[4 * N + n] = c[4];
    }
    double* H = Hs + (long long)rks * 8 * N;
  #pragma unroll
    for (int k = 0; k < 8; ++k) H[k * N + n] = (c[k] - qs[k]) / adt;
    double* HA = HsA + (long long)rks * 3 * N;
  #pragma unroll
    for (int k = 0; k < 3; ++k) HA[k * N + n] = (a[k] - as[k]) / adt;
    double* HB = HsB + (long long)rks * 2 * N;
    HB[n] = (fx - fxs) / adt;
    HB[N + n] = (fy - fys) / adt;
    double p[8];
    con2pri(P, p, c);
  #pragma unroll
    for (int k = 0; k < 8; ++k) prim[k * N + n] = p[k];
  }
};

// ---------------------------------------------------------------- shock detector
// ShockDetector (flux.cpp:5-76): fast speed per cell, chi~ (4.40), chi = 3x3 max (4.41), as
// one tiled kernel: the fast speed c_f on the tile plus a halo of 2 (shared memory), chi~ on
// the halo-1 ring, chi on the tile.  Q is read once and only eta is written (72 B/cell);
// the discrete adjoint also has chi~ of every cell stored (chit, 8 B/cell more).
// A staged halo position p holds the value of its mapped cell cid(p), as the reference's
// ghost copies do: for a periodic direction the image has the same neighbourhood, so the
// value is evaluated at p itself; for a transmissive one it is evaluated at the clamped
// position, which lies in the same tile.
constexpr int STX = 32, STY = 16, SHX = STX + 4, SHY = STY + 4, SCX = STX + 2, SCY = STY + 2;
template <bool kOpen, bool kFast>
struct k_shock {
  IMEX_BOUNDS(kThreads, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams Pin, const double* __restrict__ Q,
                                                       double* __restrict__ eta, double* __restrict__ chit) {
    const DevParams P = bc_params<kOpen>(Pin);
    const long long N = P.N;
    __shared__ double cf[SHY * SHX];  // c_f at (x0 - 2 + sx, y0 - 2 + sy)
    __shared__ double ch[SCY * SCX];  // chi~ at (x0 - 1 + px, y0 - 1 + py)
    // fast arithmetic: vx, vy of the staged cells (the exact form divides at each use)
    __shared__ double svx[kFast ? SHY * SHX : 1], svy[kFast ? SHY * SHX : 1];
    const int x0 = blockIdx.x * STX, y0 = blockIdx.y * STY;
    {  // each thread's cells of the halo-2 tile, every load before the first division
      constexpr int KC = (SHY * SHX + kThreads - 1) / kThreads;
      double c[KC][8];
  #pragma unroll
      for (int k = 0; k < KC; ++k) {
        const int q = threadIdx.x + k * kThreads;
        const int qq = q < SHY * SHX ? q : SHY * SHX - 1;  // past the end: a staged cell, loaded again
        load_cell<8>(Q, N, cid(P, x0 - 2 + qq % SHX, y0 - 2 + qq / SHX), c[k]);
      }
  #pragma unroll
      for (int k = 0; k < KC; ++k) {
        const int q = threadIdx.x + k * kThreads;
        if (q < SHY * SHX) {
          if constexpr (kFast) {
            // one reciprocal of rho per staged cell; the velocities stay in shared memory for
            // the divergence of the ring
            const double ir = 1.0 / c[k][0];
            const double vx = c[k][1] * ir, vy = c[k][2] * ir, vz = c[k][3] * ir;
            const double B2 = c[k][5] * c[k][5] + c[k][6] * c[k][6] + c[k][7] * c[k][7];
            const double e = (c[k][4] - 0.5 * c[k][0] * (vx * vx + vy * vy + vz * vz) - 0.5 * B2) * ir;
            const double p = eos_p(P, c[k][0], e);
            const double a2 = P.eos_type == IMEX_IDEAL_GAS ? P.gamma * p * ir : eos_a2(P, c[k][0], p);
            cf[q] = sqrt(a2 + B2 * ir);
            svx[q] = vx;
            svy[q] = vy;
          } else {
            const double p = pressure_of(P, c[k]);
            const double a2 = eos_a2(P, c[k][0], p);
            const double cA2 = (c[k][5] * c[k][5] + c[k][6] * c[k][6] + c[k][7] * c[k][7]) / c[k][0];
            cf[q] = sqrt(a2 + cA2);
          }
        }
      }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < SCY * SCX; q += kThreads) {
      int gi = x0 - 1 + q % SCX, gj = y0 - 1 + q / SCX;
      if (P.xclamp) gi = gi < 0 ? 0 : (gi >= P.nx ? P.nx - 1 : gi);
      if (P.yclamp) gj = gj < 0 ? 0 : (gj >= P.ny ? P.ny - 1 : gj);
      const int sx = gi - x0 + 2, sy = gj - y0 + 2;  // within [1, SHX - 2] x [1, SHY - 2]
      double m = 1.0e300;
      for (int di = -1; di <= 1; di++)
        for (int dj = -1; dj <= 1; dj++) {
          double v = cf[(sy + dj) * SHX + sx + di];
          if (v < m) m = v;
        }
      double div_u;
      if constexpr (kFast) {
        // the staged neighbours hold the same (wrapped or clamped) cells as cid's maps
        const int o = sy * SHX + sx;
        div_u = (svx[o + 1] - svx[o - 1]) * (0.5 / P.dx) + (svy[o + SHX] - svy[o - SHX]) * (0.5 / P.dy);
      } else {
        long long xp = cid(P, gi + 1, gj), xm = cid(P, gi - 1, gj), yp = cid(P, gi, gj + 1), ym = cid(P, gi, gj - 1);
        // every load before the first division
        const double mxp = __ldg(Q + N + xp), rxp = __ldg(Q + xp), mxm = __ldg(Q + N + xm), rxm = __ldg(Q + xm);
        const double myp = __ldg(Q + 2 * N + yp), ryp = __ldg(Q + yp), mym = __ldg(Q + 2 * N + ym), rym = __ldg(Q + ym);
        div_u = (mxp / rxp - mxm / rxm) / (2.0 * P.dx) + (myp / ryp - mym / rym) / (2.0 * P.dy);
      }
      double num = P.hmin * div_u + P.shock_kappa1 * m;
      double den = P.shock_kappa1 * m;
      double qv = -num / den;
      double mx = (0.0 < qv) ? qv : 0.0;
      ch[q] = (mx < 1.0) ? mx : 1.0;
      // chi~ of the tile's own cells, when asked for (chit != nullptr)
      const int lx = q % SCX - 1, ly = q / SCX - 1;
      if (chit && lx >= 0 && lx < STX && ly >= 0 && ly < STY && x0 + lx < P.nx && y0 + ly < P.ny)
        chit[(long long)(y0 + ly) * P.nx + (x0 + lx)] = ch[q];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < STX * STY; q += kThreads) {
      const int lx = q % STX, ly = q / STX, i = x0 + lx, j = y0 + ly;
      if (i >= P.nx || j >= P.ny) continue;
      double m = 0.0;
      for (int di = -1; di <= 1; di++)
        for (int dj = -1; dj <= 1; dj++) {
          double v = ch[(ly + 1 + dj) * SCX + lx + 1 + di];
          if (v > m) m = v;
        }
      eta[(long long)j * P.nx + i] = m;
    }
  }
};

// ---------------------------------------------------------------- diagnostics
// face FV div (StaggerCT; a transmissive direction's first column / row differences against
// its boundary face), central div of cell B over the neighbour map, reference cell metric
// (imex_subsystems.cpp:646-654), max |central div|
__global__ void k_divergence(DevParams P, const double* __restrict__ ucon, const double* __restrict__ bx,
                             const double* __restrict__ by, BoundaryLines L, double* __restrict__ partial) {
  const long long N = P.N;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  double m = 0.0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N; n += (long long)gridDim.x * blockDim.x) {
    int i, j;
    cell_of(P, n, i, j);
    const double bxm = (P.xclamp && i == 0) ? L.bx[j] : bx[cid(P, i - 1, j)];
    const double bym = (P.yclamp && j == 0) ? L.by[i] : by[cid(P, i, j - 1)];
    double d = (bx[n] - bxm) / P.dx + (by[n] - bym) / P.dy;
    v[0] += P.dx * P.dy * d * d;
    const double* B5 = ucon + 5 * N;
    const double* B6 = ucon + 6 * N;
    double cx = (B5[cid(P, i + 1, j)] - B5[cid(P, i - 1, j)]) / (2.0 * P.dx);
    double cy = (B6[cid(P, i, j + 1)] - B6[cid(P, i, j - 1)]) / (2.0 * P.dy);
    double c = cx + cy;
    v[1] += P.dx * P.dy * c * c;
    double rx = i == 0 ? (B5[cid(P, i + 1, j)] - B5[n]) / P.dx
                       : (i == P.nx - 1 ? (B5[n] - B5[cid(P, i - 1, j)]) / P.dx : cx);
    double ry = j == 0 ? (B6[cid(P, i, j + 1)] - B6[n]) / P.dy
                       : (j == P.ny - 1 ? (B6[n] - B6[cid(P, i, j - 1)]) / P.dy : cy);
    double r = rx + ry;
    v[2] += P.dx * P.dy * r * r;
    m = fmax(m, fabs(c));
  }
  v[3] = 0.0;
  block_reduce(v, FSum(), 0.0);
  double mm[1] = {m};
  block_reduce(mm, FMax(), 0.0);
  if (threadIdx.x == 0) {
    partial[blockIdx.x * 4 + 0] = v[0];
    partial[blockIdx.x * 4 + 1] = v[1];
    partial[blockIdx.x * 4 + 2] = v[2];
    partial[blockIdx.x * 4 + 3] = mm[0];
  }
}
__global__ void k_min_pressure(DevParams P, const double* __restrict__ prim, double* __restrict__ partial) {
  double m[1] = {INFINITY};
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < P.N; n += (long long)gridDim.x * blockDim.x)
    m[0] = fmin(m[0], prim[4 * P.N + n]);
  block_reduce(m, FMin(), INFINITY);
  if (threadIdx.x == 0) partial[blockIdx.x] = m[0];
}

// pressure and enthalpy of Qe (the planes k_stage_combine produces)
__global__ void k_qe_derived(DevParams P, const double* __restrict__ Qe, double* __restrict__ pe,
                             double* __restrict__ hQe) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= P.N) return;
  double q[8];
  load_cell<8>(Qe, P.N, n, q);
  double e = calecon(q);
  double p = eos_p(P, q[0], e);
  pe[n] = p;
  hQe[n] = e + p / q[0];
}
// Newton Jacobian diagonal V_slope(p_freeze, rho) (config.hpp:236-239)
__global__ void k_vslope(DevParams P, const DevScalars* __restrict__ sc, const double* __restrict__ pf,
                         const double* __restrict__ ucon, double* __restrict__ vdiag) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= P.N) return;
  vdiag[n] = V_slope(P, sc->Mbig, pf[n], ucon[n]);
}

}  // namespace

// ================================================================ launchers
#define LAUNCH_CHECK(ctx, what)                                         \
  do {                                                                  \
    cudaError_t e_ = cudaGetLastError();                                \
    if (e_ != cudaSuccess) return cuda_check(ctx, e_, what);            \
  } while (0)
// algorithmic bytes of a launch family: `vals` doubles moved per cell
#define BYTES(vals) ((double)(vals) * 8.0 * (double)ctx->N)

imex_status launch_step_prologue(imex_ctx* ctx) {
  const DevParams& P = ctx->P;
  int nblk = blocks_for(P.N);
  if (nblk > ctx->max_blocks) nblk = ctx->max_blocks;
  prof_begin(ctx);
  if (P.fast) launch<k_step_reduce<true>>(ctx, nblk, kThreads, 0, ctx->stream, P, ctx->prim, ctx->partial);
  else launch<k_step_reduce<false>>(ctx, nblk, kThreads, 0, ctx->stream, P, ctx->prim, ctx->partial);
  LAUNCH_CHECK(ctx, "k_step_reduce");
  launch<k_step_finalize>(ctx, 1, kThreads, 0, ctx->stream, P, ctx->partial, nblk, ctx->sc);
  LAUNCH_CHECK(ctx, "k_step_finalize");
  prof_end(ctx, F_PROLOGUE_REDUCE, BYTES(8), 2);
  prof_begin(ctx);
  launch<k_cons_from_prim>(ctx, blocks_for(P.N), kThreads, 0, ctx->stream, P, ctx->prim, ctx->cons, ctx->cons_n);
  LAUNCH_CHECK(ctx, "k_cons_from_prim");
  const long long plane = (long long)ctx->N;
  cudaError_t e = copy_d2d(ctx, ctx->bx_n, ctx->bx, plane);
  if (e == cudaSuccess) e = copy_d2d(ctx, ctx->by_n, ctx->by, plane);
  if (e == cudaSuccess) e = copy_d2d(ctx, ctx->A_snap, ctx->A, 3 * plane);
  if (e == cudaSuccess && P.xclamp) e = copy_d2d(ctx, ctx->bl.bx_n, ctx->bl.bx, P.ny);
  if (e == cudaSuccess && P.yclamp) e = copy_d2d(ctx, ctx->bl.by_n, ctx->bl.by, P.nx);
  prof_end(ctx, F_CONS_FROM_PRIM, BYTES(24 + 10), 1);
  return cuda_check(ctx, e, "step snapshot copies");
}

imex_status launch_qe_derived(imex_ctx* ctx) {
  prof_begin(ctx);
  k_qe_derived<<<blocks_for(ctx->P.N), kThreads, 0, ctx->stream>>>(ctx->P, ctx->Qe, ctx->pe, ctx->hQe);
  LAUNCH_CHECK(ctx, "k_qe_derived");
  prof_end(ctx, F_COMBINE, BYTES(10), 1);
  return IMEX_OK;
}
imex_status launch_vslope(imex_ctx* ctx) {
  k_vslope<<<blocks_for(ctx->P.N), kThreads, 0, ctx->stream>>>(ctx->P, ctx->sc, ctx->pf, ctx->cons, ctx->vdiag);
  LAUNCH_CHECK(ctx, "k_vslope");
  return IMEX_OK;
}

imex_status launch_cons_from_prim(imex_ctx* ctx) {
  launch<k_cons_from_prim>(ctx, blocks_for(ctx->P.N), kThreads, 0, ctx->stream, ctx->P, ctx->prim, ctx->cons, nullptr);
  LAUNCH_CHECK(ctx, "k_cons_from_prim");
  return IMEX_OK;
}
imex_status launch_prim_from_cons(imex_ctx* ctx) {
  k_prim_from_cons<<<blocks_for(ctx->P.N), kThreads, 0, ctx->stream>>>(ctx->P, ctx->cons, ctx->prim);
  LAUNCH_CHECK(ctx, "k_prim_from_cons");
  return IMEX_OK;
}

// Butcher tableaux of main.cpp:269-319
void tableau(int RKs, double ae[kMaxRK][kMaxRK], double ai[kMaxRK][kMaxRK]) {
  for (int r = 0; r < kMaxRK; ++r)
    for (int c = 0; c < kMaxRK; ++c) ae[r][c] = ai[r][c] = 0.0;
  if (RKs == 1) {
    ai[0][0] = 1.0;
  } else if (RKs == 2) {
    double bb = 1.0 - 1.0 / sqrt(2.0), cc = 1.0 / (2.0 * bb);
    ae[1][0] = cc;
    ai[0][0] = bb;
    ai[1][0] = 1 - bb;
    ai[1][1] = bb;
  } else {
    double r12 = 0.5, r13 = 1.0 / 3.0, r14 = 1.0 / 4.0;
    ae[1][0] = r12;
    ae[2][0] = r12;
    ae[2][1] = r12;
    ai[0][0] = r14;
    ai[1][1] = r14;
    ai[2][0] = r13;
    ai[2][1] = r13;
    ai[2][2] = r13;
  }
}

imex_status launch_stage_combine(imex_ctx* ctx, int rks) {
  double ae[kMaxRK][kMaxRK], ai[kMaxRK][kMaxRK];
  tableau(ctx->P.RKs, ae, ai);
  Tableau T{};
  for (int r = 0; r < kMaxRK; ++r) {
    T.ae[r] = ae[rks][r];
    T.ai[r] = ai[rks][r];
  }
  T.aii = ai[rks][rks];
  prof_begin(ctx);
  static_assert(kMaxRK == 3, "one k_stage_combine instance per stage index");
  const int nb = blocks_for(ctx->P.N);
  // the A form's viscosity maxima come with the combination while one pair per CTA fits
  // the partial buffer; otherwise the magnetic sub-system takes them in its own pass
  const bool g = ctx->P.magfield == IMEX_PotentialA && 2LL * nb <= ctx->partial_len;
  auto combine = [&](auto k) {
    using K = decltype(k);
    launch<K>(ctx, nb, kThreads, 0, ctx->stream, ctx->P, T, ctx->sc, ctx->cons_n, ctx->Hs, ctx->bx_n, ctx->by_n,
              ctx->HsB, ctx->A_snap, ctx->HsA, ctx->Qe, ctx->Qs, ctx->bxQe, ctx->byQe, ctx->bxQs, ctx->byQs, ctx->A_s,
              ctx->A_e, ctx->A, ctx->pe, ctx->hQe, ctx->partial);
  };
  if (g) {
    if (rks == 0) combine(k_stage_combine<0, true>{});
    else if (rks == 1) combine(k_stage_combine<1, true>{});
    else combine(k_stage_combine<2, true>{});
  } else {
    if (rks == 0) combine(k_stage_combine<0, false>{});
    else if (rks == 1) combine(k_stage_combine<1, false>{});
    else combine(k_stage_combine<2, false>{});
  }
  LAUNCH_CHECK(ctx, "k_stage_combine");
  ctx->gmax_ready = false;
  if (g) {
    imex_status s = gmax_finalize(ctx, nb);
    if (s != IMEX_OK) return s;
    ctx->gmax_ready = true;
  }
  if (ctx->P.xclamp || ctx->P.yclamp) {
    launch<k_bline_combine>(ctx, blocks_for(ctx->nx > ctx->ny ? ctx->nx : ctx->ny), kThreads, 0, ctx->stream, ctx->P, T, rks,
                                                                                                   ctx->sc, ctx->bl);
    LAUNCH_CHECK(ctx, "k_bline_combine");
  }
  prof_end(ctx, F_COMBINE, BYTES(44 + 13 * rks), g ? 2 : 1);
  return IMEX_OK;
}

// full = true stores all 8 variables (the public buffer); the stage needs only 0..4
imex_status launch_reconstruct(imex_ctx* ctx, bool full) {
  const int nstore = full ? 8 : 5;
  const int nread = ctx->P.reconstate == IMEX_PrimState ? 8 : nstore;
  prof_begin(ctx);
  if (ctx->P.reconstate == IMEX_PrimState)
    IMEX_LAUNCH_BC_ARITH(ctx->P, k_reconstruct_prim, blocks_for(ctx->P.N), kThreads, 0, ctx->stream, ctx->P, ctx->Qe,
                         ctx->w, nstore);
  else
    IMEX_LAUNCH_BC_ARITH(ctx->P, k_reconstruct_var, (dim3(blocks_for(ctx->P.N), nstore)), kThreads, 0, ctx->stream,
                         ctx->P, ctx->Qe, ctx->w);
  LAUNCH_CHECK(ctx, "k_reconstruct");
  prof_end(ctx, F_RECON, BYTES(nread + 4 * nstore), 1);
  return IMEX_OK;
}

// form 0: RusanovC_Update; 1: Pressure_flux_Update; 2: Energy_flux_Update (flux.cpp:186-200)
imex_status launch_flux_update(imex_ctx* ctx, int form) {
  const dim3 nb((ctx->nx + FTX - 1) / FTX, (ctx->ny + FTY - 1) / FTY);
  prof_begin(ctx);
  const bool open = ctx->P.xclamp || ctx->P.yclamp;
  if (form == 1)
    IMEX_LAUNCH_BC_ARITH(ctx->P, k_flux_pres, nb, FNT, 0, ctx->stream, ctx->P, ctx->sc, ctx->w, ctx->Qs, ctx->cons);
  else if (form == 2 && open)  // the energy formula's flux keeps the reference's operation order
    launch<k_flux_mag<2, true, false>>(ctx, nb, FNT, 0, ctx->stream, ctx->P, ctx->sc, ctx->w, ctx->Qs, ctx->cons);
  else if (form == 2)
    launch<k_flux_mag<2, false, false>>(ctx, nb, FNT, 0, ctx->stream, ctx->P, ctx->sc, ctx->w, ctx->Qs, ctx->cons);
  else
    IMEX_LAUNCH_BC_ARITH(ctx->P, k_flux_conv, nb, FNT, 0, ctx->stream, ctx->P, ctx->sc, ctx->w, ctx->Qs, ctx->cons);
  LAUNCH_CHECK(ctx, "flux update");
  prof_end(ctx, form ? F_FLUX_PRES : F_FLUX_CONV, BYTES(form ? 33 : 30), 1);
  return IMEX_OK;
}
// the flux of the implicit formula of this context (main.cpp:469-476)
int second_flux_form(const imex_ctx* ctx) { return ctx->P.formula == IMEX_EnergyFormula ? 2 : 1; }

// variant: 0 Staggered_CT_Consistent, 1 Unstaggered_CT_Consistent, 2 Staggered_CT, 3 Unstaggered_CT
imex_status launch_ct(imex_ctx* ctx, int variant) {
  const DevParams& P = ctx->P;
  int nb = blocks_for(P.N);
  cudaStream_t s = ctx->stream;
  prof_begin(ctx);
  if (variant == 0 || variant == 1) {
    launch<k_ct_corner>(ctx, nb, kThreads, 0, s, P, ctx->Fx, -1.0, ctx->Fy, 1.0, ctx->cons, ctx->Epp, ctx->bl);
    LAUNCH_CHECK(ctx, "k_ct_corner");
  } else if (variant == 2) {
    if (P.reconstate == IMEX_PrimState) IMEX_LAUNCH_BC_ARITH(P, k_reconstruct_prim, nb, kThreads, 0, s, P, ctx->cons, ctx->w, 8);
    else IMEX_LAUNCH_BC_ARITH(P, k_reconstruct_var, (dim3(nb, 8)), kThreads, 0, s, P, ctx->cons, ctx->w);
    LAUNCH_CHECK(ctx, "k_reconstruct(u_con)");
    launch<k_ct_legacy_faces>(ctx, nb, kThreads, 0, s, P, ctx->w, ctx->chit, ctx->Et);
    LAUNCH_CHECK(ctx, "k_ct_legacy_faces");
    launch<k_ct_corner>(ctx, nb, kThreads, 0, s, P, ctx->chit, 1.0, ctx->Et, 1.0, ctx->cons, ctx->Epp, ctx->bl);
    LAUNCH_CHECK(ctx, "k_ct_corner");
  }
  if (variant == 0 || variant == 2) {
    launch<k_ct_faces>(ctx, nb, kThreads, 0, s, P, ctx->sc, ctx->Epp, ctx->bxQs, ctx->byQs, ctx->bx, ctx->by, ctx->cons,
                                       ctx->bl);
    LAUNCH_CHECK(ctx, "k_ct_faces");
  } else {
    if (variant == 1) launch<k_ct_unstag_A>(ctx, nb, kThreads, 0, s, P, ctx->sc, ctx->Epp, ctx->A_s, ctx->A, ctx->bl);
    else launch<k_ct_unstag_legacy_A>(ctx, nb, kThreads, 0, s, P, ctx->sc, ctx->cons, ctx->A_s, ctx->A);
    LAUNCH_CHECK(ctx, "k_ct_unstag_A");
    launch<k_curl_Az>(ctx, nb, kThreads, 0, s, P, ctx->A, ctx->cons);
    LAUNCH_CHECK(ctx, "k_curl_Az");
  }
  // corner EMF 8 + faces/cell B 7 (consistent); legacy variants add the reconstruction of u_con
  prof_end(ctx, F_CT, BYTES(variant == 0 ? 15 : (variant == 1 ? 14 : (variant == 2 ? 15 + 40 + 22 : 17))), (variant == 0 ? 2 : (variant == 1 ? 3 : (variant == 2 ? 4 : 2))));
  return IMEX_OK;
}

imex_status launch_stage_derivative(imex_ctx* ctx, int rks) {
  prof_begin(ctx);
  launch<k_stage_derivative>(ctx, blocks_for(ctx->P.N), kThreads, 0, ctx->stream, 
      ctx->P, rks, ctx->sc, ctx->cons, ctx->Qs, ctx->A, ctx->A_s, ctx->bx, ctx->bxQs, ctx->by, ctx->byQs, ctx->Bsave,
      ctx->Hs, ctx->HsA, ctx->HsB, ctx->prim);
  LAUNCH_CHECK(ctx, "k_stage_derivative");
  if (ctx->P.xclamp || ctx->P.yclamp) {
    launch<k_bline_derivative>(ctx, blocks_for(ctx->nx > ctx->ny ? ctx->nx : ctx->ny), kThreads, 0, ctx->stream, 
        ctx->P, rks, ctx->sc, ctx->bl);
    LAUNCH_CHECK(ctx, "k_bline_derivative");
  }
  prof_end(ctx, F_DERIVATIVE, BYTES(47), 1);
  return IMEX_OK;
}

imex_status launch_shock(imex_ctx* ctx, const double* Q, double* eta) {
  const DevParams& P = ctx->P;
  const dim3 nb((P.nx + STX - 1) / STX, (P.ny + STY - 1) / STY);
  prof_begin(ctx);
  IMEX_LAUNCH_BC_ARITH(P, k_shock, nb, kThreads, 0, ctx->stream, P, Q, eta, ctx->keep_shock_chit ? ctx->chit : nullptr);
  LAUNCH_CHECK(ctx, "shock detector");
  prof_end(ctx, F_SHOCK, BYTES(9), 1);
  return IMEX_OK;
}

imex_status launch_divergence(imex_ctx* ctx, double* out4) {
  const DevParams& P = ctx->P;
  int nb = blocks_for(P.N);
  if (nb > ctx->max_blocks) nb = ctx->max_blocks;
  k_divergence<<<nb, kThreads, 0, ctx->stream>>>(P, ctx->cons, ctx->bx, ctx->by, ctx->bl, ctx->partial);
  LAUNCH_CHECK(ctx, "k_divergence");
  std::vector<double> h((size_t)nb * 4);
  cudaError_t e = cudaMemcpyAsync(h.data(), ctx->partial, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "divergence readback");
  double s0 = 0, s1 = 0, s2 = 0, m = 0;
  for (int b = 0; b < nb; ++b) {
    s0 += h[b * 4 + 0];
    s1 += h[b * 4 + 1];
    s2 += h[b * 4 + 2];
    m = fmax(m, h[b * 4 + 3]);
  }
  out4[0] = sqrt(s0);
  out4[1] = sqrt(s1);
  out4[2] = sqrt(s2);
  out4[3] = m;
  return IMEX_OK;
}

// out[4 c + q] for component c = central, rusanov, tilde, total and q = L2(Ez), max|Ez|,
// L2(dB/dt), max|dB/dt| (the four [CT-DIAG] lines).  Uses the reconstruction buffer and
// stage work planes, which only the inside of a stage reads.
imex_status launch_ct_diag(imex_ctx* ctx, double* out16) {
  const DevParams& P = ctx->P;
  const int nb = blocks_for(P.N);
  cudaStream_t s = ctx->stream;
  double *cp0 = ctx->chit, *c0p = ctx->Et, *rp0 = ctx->Epp, *r0p = ctx->vscale;
  if (P.reconstate == IMEX_PrimState) IMEX_LAUNCH_BC_ARITH(P, k_reconstruct_prim, nb, kThreads, 0, s, P, ctx->cons, ctx->w, 8);
  else IMEX_LAUNCH_BC_ARITH(P, k_reconstruct_var, (dim3(nb, 8)), kThreads, 0, s, P, ctx->cons, ctx->w);
  k_ct_diag_faces<<<nb, kThreads, 0, s>>>(P, ctx->w, cp0, c0p, rp0, r0p);
  int nred = nb < ctx->max_blocks ? nb : ctx->max_blocks;
  k_ct_diag_stats<<<nred, kThreads, 0, s>>>(P, cp0, c0p, rp0, r0p, ctx->cons, ctx->partial);
  LAUNCH_CHECK(ctx, "CT EMF diagnostics");
  std::vector<double> h((size_t)nred * 16);
  cudaError_t e = cudaMemcpyAsync(h.data(), ctx->partial, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_check(ctx, e, "CT EMF diagnostics readback");
  double sum[8] = {0, 0, 0, 0, 0, 0, 0, 0}, mx[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = 0; b < nred; ++b)
    for (int k = 0; k < 8; ++k) {
      sum[k] += h[(size_t)b * 16 + k];
      mx[k] = fmax(mx[k], h[(size_t)b * 16 + 8 + k]);
    }
  for (int c = 0; c < 4; ++c) {
    out16[4 * c + 0] = sqrt(sum[c]);
    out16[4 * c + 1] = mx[c];
    out16[4 * c + 2] = sqrt(sum[4 + c]);
    out16[4 * c + 3] = mx[4 + c];
  }
  return IMEX_OK;
}

imex_status launch_min_pressure(imex_ctx* ctx, double* pmin) {
  const DevParams& P = ctx->P;
  int nb = blocks_for(P.N);
  if (nb > ctx->max_blocks) nb = ctx->max_blocks;
  k_min_pressure<<<nb, kThreads, 0, ctx->stream>>>(P, ctx->prim, ctx->partial);
  LAUNCH_CHECK(ctx, "k_min_pressure");
  std::vector<double> h(nb);
  cudaError_t e = cudaMemcpyAsync(h.data(), ctx->partial, nb * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "min pressure readback");
  double m = INFINITY;
  for (int b = 0; b < nb; ++b) m = fmin(m, h[b]);
  *pmin = m;
  return IMEX_OK;
}


// queue the copy of this translation unit's EOS flag into pinned host memory (no wait)
imex_status eos_flag_stage_enqueue(imex_ctx* ctx, int* host_flag) {
  return cuda_check(ctx, cudaMemcpyFromSymbolAsync(host_flag, d_eos_flag, sizeof(int), 0, cudaMemcpyDeviceToHost,
                                                   ctx->stream),
                    "eos flag");
}
imex_status eos_flag_stage(imex_ctx* ctx, int* flag, bool reset) {
  cudaError_t e = cudaMemcpyFromSymbolAsync(&ctx->h_red[0], d_eos_flag, sizeof(int), 0, cudaMemcpyDeviceToHost,
                                            ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "eos flag");
  int v = 0;
  memcpy(&v, &ctx->h_red[0], sizeof(int));
  *flag = v;
  if (reset && v) {
    static const int zero = 0;
    e = cudaMemcpyToSymbolAsync(d_eos_flag, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  }
  return cuda_check(ctx, e, "eos flag reset");
}

}  // namespace imex
