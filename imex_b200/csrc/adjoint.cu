// Discrete adjoint of the IMEX-RK step (imex_adjoint_run / imex_adjoint_vjp).
//
// The forward step is a chain of sub-steps (main.cpp:335-561); its adjoint runs the chain
// backwards, each sub-step contributing its vector-Jacobian product:
//   * stencil sub-steps (magnetic right-hand side, CollectMagFluxes, pressure right-hand
//     side, momentum, DefinitionofU or ConservationofU, the CT corner EMF, the frozen
//     coefficients): the shared cell functions (cells.cuh) evaluated in dual numbers with L
//     inputs seeded per pass, the products scattered to the inputs;
//   * the explicit fluxes: per face, the Rusanov flux in dual numbers, then the
//     reconstruction per variable and direction (ConsState) or per stencil cell with its 8
//     conserved planes seeded through con2pri, recon and pri2con (PrimState);
//   * each implicit solve A(theta) x = b: one transposed GMRES solve A^T mu = lambda_x on
//     the assembled transposed stencil, lambda_b = mu, lambda_theta -= mu^T d(A x)/d theta;
//     the nested Newton is differentiated at its converged p through its active set
//     (J = diag(V_slope(p)) + T, with the Cor.1 slope Mbig and its dependence on min b);
//   * the GLF maxima (a_max, B_max, vx/vy_max) pass their adjoints to the cell that
//     attains each maximum;
//   * the linear stage combination, stage derivative and CT face update by hand.
// Across steps: checkpoints every K steps, the steps of a segment recomputed from its
// checkpoint, and each step recomputed once more with its sub-step states kept.
//
// Supported: PressureFormula, StaggerCT (B-form magnetic solve), ConsState or PrimState
// reconstruction, ideal gas, GLF, any pressure viscosity, fixed dt, FP64,
// either energy update, Energy_Modify on or off; other configurations return
// IMEX_ERR_UNSUPPORTED.
#include <cstdio>
#include <cstring>
#include <functional>
#include <vector>

#include "cells.cuh"
#include "imex_internal.h"

namespace imex {
namespace {

constexpr int kAT = 128;  // threads per block of the dual-number kernels
inline int ablocks(long long n) { return (int)((n + kAT - 1) / kAT); }

#define ACHECK(ctx, what)                                                     \
  do {                                                                        \
    cudaError_t e_ = cudaGetLastError();                                      \
    if (e_ != cudaSuccess) return cuda_check(ctx, e_, what);                  \
  } while (0)

// ------------------------------------------------------------------ generic cell VJP
// A cell function reads arrays a < kMaxArr through ld(a, k, m).  Array a is seeded on the
// planes whose bits are set in pmask[a] and at the neighbours of the 3x3 neighbourhood whose
// bits are set in mask[a] (bit o = neighbour nb[o]); its adjoint accumulates into lam[a].
// The masks must cover every plane and neighbour the cell function reads of that array.
// Scalars (at most 2) are seeded after the arrays.
constexpr int kMaxArr = 5;
constexpr unsigned OFS_C = 1u << NB_C;
constexpr unsigned OFS_CROSS = OFS_C | (1u << NB_E) | (1u << NB_W) | (1u << NB_N) | (1u << NB_S);
constexpr unsigned OFS_ALL = 0x1FFu;
constexpr unsigned OFS_NO_SW = OFS_ALL & ~(1u << NB_SW);
struct CellVjp {
  const double* in[kMaxArr];
  double* lam[kMaxArr];
  unsigned pmask[kMaxArr];  // seeded planes
  unsigned mask[kMaxArr];   // seeded neighbours
  const double* lam_out[8];  // adjoint of each output (one plane each)
  double sval[2];
  double* lam_s;
  double h, sx, sy;
};

template <int L>
struct SeedLoad {
  const CellVjp& A;
  const long long* nb;
  long long N;
  int base[kMaxArr];
  int q0;
  __device__ __forceinline__ Dual<L> operator()(int a, int k, long long m) const {
    Dual<L> r(__ldg(A.in[a] + (long long)k * N + m));
    if ((A.pmask[a] >> k) & 1u) {
      const int kk = __popc(A.pmask[a] & ((1u << k) - 1u));
      const unsigned mask = A.mask[a];
      int oi = -1;
#pragma unroll
      for (int o = 0; o < 9; ++o)
        if (((mask >> o) & 1u) && nb[o] == m) oi = o;
      if (oi >= 0) {
        const int l = base[a] + kk * __popc(mask) + __popc(mask & ((1u << oi) - 1u)) - q0;
#pragma unroll
        for (int ll = 0; ll < L; ++ll)
          if (ll == l) r.d[ll] = 1.0;
      }
    }
    return r;
  }
};

template <int L, class Fn>
__global__ void __launch_bounds__(kAT) k_cell_vjp(DevParams P, CellVjp A, Fn fn) {
  __shared__ double s_acc[2];
  if (threadIdx.x < 2) s_acc[threadIdx.x] = 0.0;
  __syncthreads();
  const long long N = P.N;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n < N) {
    double lo[Fn::NOUT];
    bool any = false;
#pragma unroll
    for (int j = 0; j < Fn::NOUT; ++j) {
      lo[j] = A.lam_out[j] ? A.lam_out[j][n] : 0.0;
      any = any || lo[j] != 0.0;
    }
    if (any) {
      long long nb[9];
      neighbours(P, n, nb);
      SeedLoad<L> ld{A, nb, N, {0, 0, 0, 0, 0}, 0};
      int nin = 0;
      for (int a = 0; a < kMaxArr; ++a) {
        ld.base[a] = nin;
        nin += __popc(A.pmask[a]) * __popc(A.mask[a]);
      }
      const int ntot = nin + Fn::NS;
      for (int q0 = 0; q0 < ntot; q0 += L) {
        ld.q0 = q0;
        Dual<L> sc[Fn::NS > 0 ? Fn::NS : 1];
#pragma unroll
        for (int s = 0; s < Fn::NS; ++s) {
          sc[s] = Dual<L>(A.sval[s]);
          const int l = nin + s - q0;
#pragma unroll
          for (int ll = 0; ll < L; ++ll)
            if (ll == l) sc[s].d[ll] = 1.0;
        }
        Dual<L> out[Fn::NOUT];
        fn(P, A, nb, sc, ld, out);
#pragma unroll
        for (int l = 0; l < L; ++l) {
          const int q = q0 + l;
          if (q >= ntot) break;
          double c = 0.0;
#pragma unroll
          for (int j = 0; j < Fn::NOUT; ++j) c += lo[j] * out[j].d[l];
          if (c == 0.0) continue;
          if (q >= nin) {
            atomicAdd(&s_acc[q - nin], c);
            continue;
          }
          int a = 0;
          while (a + 1 < kMaxArr && q >= ld.base[a + 1]) ++a;
          const unsigned mask = A.mask[a], pmask = A.pmask[a];
          const int cnt = __popc(mask), r = q - ld.base[a];
          int kr = r / cnt, rank = r % cnt, o = 0, k = 0;
          for (; o < 9; ++o)
            if ((mask >> o) & 1u) {
              if (rank == 0) break;
              --rank;
            }
          for (; k < 8; ++k)
            if ((pmask >> k) & 1u) {
              if (kr == 0) break;
              --kr;
            }
          atomicAdd(A.lam[a] + (long long)k * N + nb[o], c);
        }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < Fn::NS && s_acc[threadIdx.x] != 0.0) atomicAdd(A.lam_s + threadIdx.x, s_acc[threadIdx.x]);
}

struct FnMagRhs {
  static constexpr int NOUT = 3, NS = 0;
  template <class S, class Ld>
  __device__ void operator()(const DevParams& P, const CellVjp& A, const long long* nb, const S*, Ld& ld,
                             S* out) const {
    mag_rhs_B_cell<S>(P, A.h, nb, ld, out);
  }
};
struct FnCollect {
  static constexpr int NOUT = 2, NS = 2;
  template <class S, class Ld>
  __device__ void operator()(const DevParams& P, const CellVjp& A, const long long* nb, const S* sc, Ld& ld,
                             S* out) const {
    collect_cell<S>(P, A.h, sc, nb, ld, out);
  }
};
struct FnPresRhs {
  static constexpr int NOUT = 1, NS = 0;
  template <class S, class Ld>
  __device__ void operator()(const DevParams& P, const CellVjp& A, const long long* nb, const S*, Ld& ld,
                             S* out) const {
    pressure_rhs_cell<S>(P, A.h, nb, ld, out);
  }
};
struct FnMomentum {
  static constexpr int NOUT = 2, NS = 0;
  template <class S, class Ld>
  __device__ void operator()(const DevParams& P, const CellVjp& A, const long long* nb, const S*, Ld& ld,
                             S* out) const {
    momentum_cell<S>(P, A.h, nb, ld, out);
  }
};
struct FnEnergyDef {
  static constexpr int NOUT = 1, NS = 0;
  template <class S, class Ld>
  __device__ void operator()(const DevParams& P, const CellVjp&, const long long* nb, const S*, Ld& ld,
                             S* out) const {
    energy_define_cell<S>(P, nb, ld, out);
  }
};
struct FnEnergyCons {
  static constexpr int NOUT = 1, NS = 0;
  template <class S, class Ld>
  __device__ void operator()(const DevParams& P, const CellVjp& A, const long long* nb, const S*, Ld& ld,
                             S* out) const {
    energy_conservation_cell<S>(P, A.h, nb, ld, out);
  }
};
struct FnCtCorner {
  static constexpr int NOUT = 1, NS = 0;
  template <class S, class Ld>
  __device__ void operator()(const DevParams& P, const CellVjp& A, const long long* nb, const S*, Ld& ld,
                             S* out) const {
    ct_corner_cell<S>(P, A.sx, A.sy, nb, ld, out);
  }
};
struct FnHh {
  static constexpr int NOUT = 1, NS = 0;
  template <class S, class Ld>
  __device__ void operator()(const DevParams& P, const CellVjp&, const long long* nb, const S*, Ld& ld,
                             S* out) const {
    hh_cell<S>(P, nb, ld, out);
  }
};
struct FnPe {
  static constexpr int NOUT = 1, NS = 0;
  template <class S, class Ld>
  __device__ void operator()(const DevParams& P, const CellVjp&, const long long* nb, const S*, Ld& ld,
                             S* out) const {
    pe_cell<S>(P, nb, ld, out);
  }
};
// fast speed of the shock detector, sqrt(a^2 + |B|^2 / rho) of Qe (flux.cpp:20-31)
struct FnShockCf {
  static constexpr int NOUT = 1, NS = 0;
  template <class S, class Ld>
  __device__ void operator()(const DevParams& P, const CellVjp&, const long long* nb, const S*, Ld& ld,
                             S* out) const {
    S c[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) c[k] = ld(0, k, nb[NB_C]);
    S p = pressure_of(P, c);
    S a2 = eos_a2(P, c[0], p);
    S cA2 = (c[5] * c[5] + c[6] * c[6] + c[7] * c[7]) / c[0];
    out[0] = sqrt(a2 + cA2);
  }
};
// conserved state of a primitive state (the step start, main.cpp:356-358)
struct FnPri2Con {
  static constexpr int NOUT = 8, NS = 0;
  template <class S, class Ld>
  __device__ void operator()(const DevParams& P, const CellVjp&, const long long* nb, const S*, Ld& ld,
                             S* out) const {
    S p[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) p[k] = ld(0, k, nb[NB_C]);
    pri2con(P, out, p);
  }
};

CellVjp cv_empty() {
  CellVjp A;
  memset(&A, 0, sizeof(A));
  return A;
}
// array a seeded on planes [k0, k0 + nk) at the neighbours in `mask`
void cv_arr(CellVjp& A, int a, const double* in, double* lam, int k0, int nk, unsigned mask) {
  A.in[a] = in;
  A.lam[a] = lam;
  A.pmask[a] = lam ? ((1u << nk) - 1u) << k0 : 0u;
  A.mask[a] = mask;
}
// array a seeded on the planes in `pmask`
void cv_arr_planes(CellVjp& A, int a, const double* in, double* lam, unsigned pmask, unsigned mask) {
  A.in[a] = in;
  A.lam[a] = lam;
  A.pmask[a] = lam ? pmask : 0u;
  A.mask[a] = mask;
}
template <int L, class Fn>
imex_status run_cell_vjp(imex_ctx* ctx, const CellVjp& A, Fn fn) {
  // unused arrays still need a readable base pointer for the value loads of the cell function
  prof_begin(ctx);
  k_cell_vjp<L, Fn><<<ablocks(ctx->P.N), kAT, 0, ctx->stream>>>(ctx->P, A, fn);
  ACHECK(ctx, "k_cell_vjp");
  prof_end(ctx, F_ADJ_CELLS, 0.0, 1);
  return IMEX_OK;
}

// ------------------------------------------------------------------ explicit fluxes
// Per face between cell n and its +x / +y neighbour m: lambda_F = (h/d)(lambda_u(m) -
// lambda_u(n)), then the Rusanov face flux in dual numbers over (QL, QR, a_max).
template <int kForm>
__global__ void __launch_bounds__(kAT) k_adj_flux(DevParams P, double h, double a_max, const double* __restrict__ w,
                                                 const double* __restrict__ ucon, const double* __restrict__ lam_u,
                                                 double* __restrict__ lam_w, double* __restrict__ lam_ucon,
                                                 double* __restrict__ lam_Qs, double* __restrict__ lam_amax) {
  constexpr int L = 6, NI = 17;
  const long long N = P.N;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double acc_a = 0.0;
  if (n < N) {
    int i, j;
    cell_of(P, n, i, j);
    for (int k = 0; k < 5; ++k) lam_Qs[k * N + n] += lam_u[k * N + n];
    for (int dir = 0; dir < 2; ++dir) {
      const long long m = dir ? cid(P, i, j + 1) : cid(P, i + 1, j);
      const double d = dir ? P.dy : P.dx;
      double lf[5];
      bool any = false;
      for (int k = 0; k < 5; ++k) {
        lf[k] = (h / d) * (lam_u[k * N + m] - lam_u[k * N + n]);
        any = any || lf[k] != 0.0;
      }
      if (!any) continue;
      const int rblk = dir ? 3 : 1, lblk = dir ? 2 : 0;  // w = [xL | xR | yL | yR] x 8 planes
      double ql[8], qr[8];
      for (int k = 0; k < 5; ++k) {
        ql[k] = w[(rblk * 8 + k) * N + n];
        qr[k] = w[(lblk * 8 + k) * N + m];
      }
      for (int k = 5; k < 8; ++k) {
        ql[k] = kForm ? ucon[k * N + n] : 0.0;
        qr[k] = kForm ? ucon[k * N + m] : 0.0;
      }
      for (int q0 = 0; q0 < NI; q0 += L) {
        Dual<L> QL[8], QR[8], am(a_max);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          QL[k] = Dual<L>(ql[k]);
          QR[k] = Dual<L>(qr[k]);
#pragma unroll
          for (int l = 0; l < L; ++l) {
            if (q0 + l == k) QL[k].d[l] = 1.0;
            if (q0 + l == 8 + k) QR[k].d[l] = 1.0;
          }
        }
#pragma unroll
        for (int l = 0; l < L; ++l)
          if (q0 + l == 16) am.d[l] = 1.0;
        Dual<L> F[5];
        face_flux<kForm>(P, QL, QR, dir, am, F);
#pragma unroll
        for (int l = 0; l < L; ++l) {
          const int q = q0 + l;
          if (q >= NI) break;
          double c = 0.0;
#pragma unroll
          for (int k = 0; k < 5; ++k) c += lf[k] * F[k].d[l];
          if (c == 0.0) continue;
          if (q == 16) {
            acc_a += c;
          } else {
            const bool left = q < 8;
            const int v = left ? q : q - 8;
            const long long cell = left ? n : m;
            if (v < 5) lam_w[((left ? rblk : lblk) * 8 + v) * N + cell] += c;
            else if (kForm) atomicAdd(lam_ucon + v * N + cell, c);
          }
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc_a += __shfl_xor_sync(0xffffffffu, acc_a, o);
  if ((threadIdx.x & 31) == 0 && acc_a != 0.0) atomicAdd(lam_amax, acc_a);
}
// reconstruction (ConsState, per variable): lambda_Q(c) += sum over the cells whose 5-point
// stencils contain c of lambda_w(cell) dw(cell)/dQ(c)
__global__ void __launch_bounds__(kAT) k_adj_recon(DevParams P, const double* __restrict__ Q,
                                                  const double* __restrict__ lam_w, double* __restrict__ lam_Q,
                                                  int nvars) {
  const long long N = P.N;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  int i, j;
    cell_of(P, n, i, j);
  const bool vortex = P.recon == IMEX_Minmod && P.vortex_minmod;
  for (int k = 0; k < nvars; ++k) {
    const double* a = Q + k * N;
    double acc = 0.0;
    for (int dir = 0; dir < 2; ++dir) {
      for (int dd = -2; dd <= 2; ++dd) {
        const long long jj = dir ? cid(P, i, j + dd) : cid(P, i + dd, j);
        const double lwl = lam_w[((dir ? 2 : 0) * 8 + k) * N + jj];
        const double lwr = lam_w[((dir ? 3 : 1) * 8 + k) * N + jj];
        if (lwl == 0.0 && lwr == 0.0) continue;
        Dual<1> u[5];
#pragma unroll
        for (int t = 0; t < 5; ++t) {
          const long long idx = dir ? cid(P, i, j + dd + t - 2) : cid(P, i + dd + t - 2, j);
          u[t] = Dual<1>(a[idx]);
          if (idx == n) u[t].d[0] = 1.0;
        }
        Dual<1> wl, wr;
        recon_1d(P.recon, u[0], u[1], u[2], u[3], u[4], wl, wr, dir ? vortex : false);
        acc += lwl * wl.d[0] + lwr * wr.d[0];
      }
    }
    lam_Q[k * N + n] += acc;
  }
}

// reconstruction (PrimState): each face state is pri2con(recon(con2pri(Q))) with every
// primitive variable reconstructed on its own (reconstruction.cpp:272-281), so a face state's
// conserved planes depend on all 8 conserved planes of each stencil cell.  lambda_Q(c) +=
// sum over the cells whose 5-point stencils contain c of lambda_w(cell) dw(cell)/dQ(c), with
// the 8 planes of Q(c) seeded at once; only the first nvars conserved planes of the face
// states carry adjoints (the fluxes take cell B from u_con).
__global__ void __launch_bounds__(kAT) k_adj_recon_prim(DevParams P, const double* __restrict__ Q,
                                                       const double* __restrict__ lam_w,
                                                       double* __restrict__ lam_Q, int nvars) {
  const long long N = P.N;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  int i, j;
  cell_of(P, n, i, j);
  const bool vortex = P.recon == IMEX_Minmod && P.vortex_minmod;
  Dual<8> dp[8];  // primitive state of cell n, seeded on its conserved planes
  {
    Dual<8> c[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      c[k] = Dual<8>(Q[k * N + n]);
      c[k].d[k] = 1.0;
    }
    con2pri(P, dp, c);
  }
  double acc[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) acc[q] = 0.0;
  for (int dir = 0; dir < 2; ++dir) {
    for (int dd = -2; dd <= 2; ++dd) {
      const long long m = dir ? cid(P, i, j + dd) : cid(P, i + dd, j);
      const double* lwl = lam_w + (long long)(dir ? 2 : 0) * 8 * N + m;
      const double* lwr = lam_w + (long long)(dir ? 3 : 1) * 8 * N + m;
      bool any = false;
      for (int k = 0; k < nvars; ++k) any = any || lwl[k * N] != 0.0 || lwr[k * N] != 0.0;
      if (!any) continue;
      double pv[5][8];
      bool seed[5];
#pragma unroll
      for (int t = 0; t < 5; ++t) {
        const long long idx = dir ? cid(P, i, j + dd + t - 2) : cid(P, i + dd + t - 2, j);
        seed[t] = idx == n;
        double c[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) c[k] = Q[k * N + idx];
        con2pri(P, pv[t], c);
      }
      Dual<8> wl[8], wr[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        Dual<8> u[5];
#pragma unroll
        for (int t = 0; t < 5; ++t) u[t] = seed[t] ? dp[k] : Dual<8>(pv[t][k]);
        recon_1d(P.recon, u[0], u[1], u[2], u[3], u[4], wl[k], wr[k], dir ? vortex : false);
      }
      Dual<8> cl[8], cr[8];
      pri2con(P, cl, wl);
      pri2con(P, cr, wr);
      for (int k = 0; k < nvars; ++k) {
        const double a = lwl[k * N], b = lwr[k * N];
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] += a * cl[k].d[q] + b * cr[k].d[q];
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 8; ++q) lam_Q[q * N + n] += acc[q];
}
// the reconstruction's adjoint for the configured reconstructed state
void adj_recon(const DevParams& P, cudaStream_t st, const double* Q, const double* lam_w, double* lam_Q) {
  const int nb = ablocks(P.N);
  if (P.reconstate == IMEX_PrimState) k_adj_recon_prim<<<nb, kAT, 0, st>>>(P, Q, lam_w, lam_Q, 5);
  else k_adj_recon<<<nb, kAT, 0, st>>>(P, Q, lam_w, lam_Q, 5);
}

// ------------------------------------------------------------------ linear sub-steps
struct Coefs {
  double ae[kMaxRK], ai[kMaxRK];
};
// stage combination (main.cpp:368-409): Qe = u^n + dt sum ae Hs, Qs = u^n + dt sum ai Hs, faces
__global__ void k_adj_combine(DevParams P, Coefs T, int rks, double dt, const double* __restrict__ lam_Qe,
                              const double* __restrict__ lam_Qs, const double* __restrict__ lam_bxQs,
                              const double* __restrict__ lam_byQs, double* __restrict__ lam_cons_n,
                              double* __restrict__ lam_Hs, double* __restrict__ lam_bx_n, double* __restrict__ lam_by_n,
                              double* __restrict__ lam_HsB) {
  const long long N = P.N;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  for (int k = 0; k < 8; ++k) {
    const double lq = lam_Qe[k * N + n], ls = lam_Qs[k * N + n];
    lam_cons_n[k * N + n] += lq + ls;
    for (int r = 0; r < rks; ++r) lam_Hs[((long long)r * 8 + k) * N + n] += T.ae[r] * dt * lq + T.ai[r] * dt * ls;
  }
  const double lbx = lam_bxQs[n], lby = lam_byQs[n];
  lam_bx_n[n] += lbx;
  lam_by_n[n] += lby;
  for (int r = 0; r < rks; ++r) {
    lam_HsB[((long long)r * 2 + 0) * N + n] += T.ai[r] * dt * lbx;
    lam_HsB[((long long)r * 2 + 1) * N + n] += T.ai[r] * dt * lby;
  }
}
// stage derivative (main.cpp:539-555): Hs = (u - Qs) / adt, HsB = (faces - faces_Qs) / adt.
// With Energy_Modify (main.cpp:528-534) u is the CT output with E += (|B|^2 - |B_save|^2) / 2
// first (bct = cell B of the CT output, bsave = cell B after the magnetic sub-system).
__global__ void k_adj_derivative(DevParams P, int rks, double adt, const double* __restrict__ lam_out,
                                 const double* __restrict__ lam_bx_out, const double* __restrict__ lam_by_out,
                                 const double* __restrict__ lam_Hs, const double* __restrict__ lam_HsB,
                                 double* __restrict__ lam5, double* __restrict__ lam_Qs, double* __restrict__ lam_bx5,
                                 double* __restrict__ lam_by5, double* __restrict__ lam_bxQs,
                                 double* __restrict__ lam_byQs, const double* __restrict__ bct,
                                 const double* __restrict__ bsave, double* __restrict__ lam_bsave) {
  const long long N = P.N;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  for (int k = 0; k < 8; ++k) {
    const double lh = lam_Hs[((long long)rks * 8 + k) * N + n] / adt;
    lam5[k * N + n] = (lam_out ? lam_out[k * N + n] : 0.0) + lh;
    lam_Qs[k * N + n] = -lh;
  }
  if (bct) {
    const double le = lam5[4 * N + n];
    for (int k = 0; k < 3; ++k) {
      lam5[(5 + k) * N + n] += le * bct[k * N + n];
      lam_bsave[k * N + n] = -le * bsave[k * N + n];
    }
  }
  const double hx = lam_HsB[((long long)rks * 2 + 0) * N + n] / adt, hy = lam_HsB[((long long)rks * 2 + 1) * N + n] / adt;
  lam_bx5[n] = (lam_bx_out ? lam_bx_out[n] : 0.0) + hx;
  lam_by5[n] = (lam_by_out ? lam_by_out[n] : 0.0) + hy;
  lam_bxQs[n] = -hx;
  lam_byQs[n] = -hy;
}
// CT face update (ct_flux.cpp:174-189): bx -= h/dy dEz, by += h/dx dEz, cell B = face averages
__global__ void k_adj_ct_faces1(DevParams P, const double* __restrict__ lam5, const double* __restrict__ lam_bx5,
                                const double* __restrict__ lam_by5, double* __restrict__ lam_bxt,
                                double* __restrict__ lam_byt, double* __restrict__ lam_bxQs,
                                double* __restrict__ lam_byQs, double* __restrict__ lam4) {
  const long long N = P.N;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  int i, j;
    cell_of(P, n, i, j);
  const long long ip = cid(P, i + 1, j), jp = cid(P, i, j + 1);
  const double bxt = lam_bx5[n] + 0.5 * lam5[5 * N + n] + 0.5 * lam5[5 * N + ip];
  const double byt = lam_by5[n] + 0.5 * lam5[6 * N + n] + 0.5 * lam5[6 * N + jp];
  lam_bxt[n] = bxt;
  lam_byt[n] = byt;
  lam_bxQs[n] += bxt;
  lam_byQs[n] += byt;
  for (int k = 0; k < 8; ++k) lam4[k * N + n] = (k == 5 || k == 6) ? 0.0 : lam5[k * N + n];
}
__global__ void k_adj_ct_faces2(DevParams P, double h, const double* __restrict__ lam_bxt,
                                const double* __restrict__ lam_byt, double* __restrict__ lam_E) {
  const long long N = P.N;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  int i, j;
    cell_of(P, n, i, j);
  const long long ip = cid(P, i + 1, j), jp = cid(P, i, j + 1);
  lam_E[n] = -(h / P.dy) * lam_bxt[n] + (h / P.dy) * lam_bxt[jp] + (h / P.dx) * lam_byt[n] - (h / P.dx) * lam_byt[ip];
}
// a += b on k planes
__global__ void k_axpy_planes(long long n_all, double* __restrict__ a, const double* __restrict__ b, double s) {
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n < n_all) a[n] += s * b[n];
}

// ------------------------------------------------------------------ shock detector
// eta = 3x3 max of chi~ (flux.cpp:60-76): the adjoint goes to the cell the forward loop kept
__global__ void k_adj_shock_max(DevParams P, const double* __restrict__ chit, const double* __restrict__ lam_eta,
                                double* __restrict__ lam_chit) {
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= P.N) return;
  const double le = lam_eta[n];
  if (le == 0.0) return;
  int i, j;
    cell_of(P, n, i, j);
  double m = 0.0;
  long long arg = -1;
  for (int di = -1; di <= 1; di++)
    for (int dj = -1; dj <= 1; dj++) {
      const long long c = cid(P, i + di, j + dj);
      const double v = chit[c];
      if (v > m) {
        m = v;
        arg = c;
      }
    }
  if (arg >= 0) atomicAdd(lam_chit + arg, le);
}
// chi~ = clamp(-(hmin div v + k1 cf_min) / (k1 cf_min), 0, 1) (flux.cpp:33-58)
__global__ void k_adj_shock_tilde(DevParams P, const double* __restrict__ Q, const double* __restrict__ cf,
                                  const double* __restrict__ lam_chit, double* __restrict__ lam_Q,
                                  double* __restrict__ lam_cf) {
  const long long N = P.N;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  const double lc = lam_chit[n];
  if (lc == 0.0) return;
  int i, j;
    cell_of(P, n, i, j);
  double m = 1.0e300;
  long long arg = -1;
  for (int di = -1; di <= 1; di++)
    for (int dj = -1; dj <= 1; dj++) {
      const long long c = cid(P, i + di, j + dj);
      const double v = cf[c];
      if (v < m) {
        m = v;
        arg = c;
      }
    }
  const long long xp = cid(P, i + 1, j), xm = cid(P, i - 1, j), yp = cid(P, i, j + 1), ym = cid(P, i, j - 1);
  const double div_u = (Q[N + xp] / Q[xp] - Q[N + xm] / Q[xm]) / (2.0 * P.dx) +
                       (Q[2 * N + yp] / Q[yp] - Q[2 * N + ym] / Q[ym]) / (2.0 * P.dy);
  const double k1 = P.shock_kappa1;
  const double q = -(P.hmin * div_u + k1 * m) / (k1 * m);
  if (!(q > 0.0 && q < 1.0)) return;  // clamped: no dependence
  const double l_div = lc * (-P.hmin / (k1 * m));
  const double l_m = lc * (P.hmin * div_u / (k1 * m * m));
  if (arg >= 0) atomicAdd(lam_cf + arg, l_m);
  const double gx = l_div / (2.0 * P.dx), gy = l_div / (2.0 * P.dy);
  atomicAdd(lam_Q + N + xp, gx / Q[xp]);
  atomicAdd(lam_Q + xp, -gx * Q[N + xp] / (Q[xp] * Q[xp]));
  atomicAdd(lam_Q + N + xm, -gx / Q[xm]);
  atomicAdd(lam_Q + xm, gx * Q[N + xm] / (Q[xm] * Q[xm]));
  atomicAdd(lam_Q + 2 * N + yp, gy / Q[yp]);
  atomicAdd(lam_Q + yp, -gy * Q[2 * N + yp] / (Q[yp] * Q[yp]));
  atomicAdd(lam_Q + 2 * N + ym, -gy / Q[ym]);
  atomicAdd(lam_Q + ym, gy * Q[2 * N + ym] / (Q[ym] * Q[ym]));
}

// ------------------------------------------------------------------ nested Newton pieces
// J-mode diagonal V_slope(p) at the converged pressure
__global__ void k_adj_vdiag(DevParams P, double Mbig, const double* __restrict__ p, const double* __restrict__ rho,
                            double* __restrict__ vd) {
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n < P.N) vd[n] = V_slope(P, Mbig, p[n], rho[n]);
}
// sum over floored cells of mu (p - p_floor): d g / d Mbig (implicit_operators.cpp:693-697)
__global__ void k_adj_mbig_sum(DevParams P, const double* __restrict__ p, const double* __restrict__ mu,
                               double* __restrict__ acc) {
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double s = 0.0;
  if (n < P.N && p[n] < P.p_floor) s = mu[n] * (p[n] - P.p_floor);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s != 0.0) atomicAdd(acc, s);
}
// min of b and the first cell attaining it
__global__ void k_adj_bmin(long long N, const double* __restrict__ b, double bmin, unsigned long long* __restrict__ idx) {
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n < N && b[n] == bmin) atomicMin(idx, (unsigned long long)n);
}
__global__ void k_min_reduce(long long N, const double* __restrict__ b, double* __restrict__ out) {
  __shared__ double sh[kAT / 32];
  double m = INFINITY;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N; n += (long long)gridDim.x * blockDim.x)
    m = fmin(m, b[n]);
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kAT / 32; ++w) m = fmin(m, sh[w]);
    sh[0] = m;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // a non-negative double orders like its bit pattern; min over blocks via a signed-safe loop
    unsigned long long* a = reinterpret_cast<unsigned long long*>(out);
    unsigned long long old = *a, assumed;
    do {
      assumed = old;
      if (__longlong_as_double((long long)assumed) <= sh[0]) break;
      old = atomicCAS(a, assumed, (unsigned long long)__double_as_longlong(sh[0]));
    } while (old != assumed);
  }
}

// ------------------------------------------------------------------ GLF maxima (step prologue)
// per-cell quantities of k_step_reduce (timestep.cpp:5-148,254-273) in the same arithmetic:
// 0 a_max (ch on the first step, v_max after), 1 B_max_x, 2 B_max_y, 3 vx_max, 4 vy_max,
// 5 cA_x, 6 cA_y (the Alfven maxima of the AlfvenSpeedp pressure viscosity)
constexpr int kGlfQ = 7;
template <class S>
__device__ __forceinline__ void glf_quantities(const DevParams& P, const S* p, bool first, S* q) {
  S B2 = p[5] * p[5] + p[6] * p[6] + p[7] * p[7];
  S B = sqrt(B2);
  S vv = sqrt(p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
  if (P.fast) {  // the fast form of k_step_reduce, operation for operation
    const S ir = 1.0 / p[0];
    if (first) {
      const S a2 = P.eos_type == IMEX_IDEAL_GAS ? P.gamma * p[4] * ir : eos_a2(P, p[0], p[4]);
      const S t = a2 + B2 * ir, tt = t * t, a4 = 4.0 * a2 * ir;
      S disc = tt - a4 * B * B;
      if (disc < 0) disc = 0;
      q[0] = vv + sqrt(0.5 * (t + sqrt(disc)));
    } else {
      q[0] = vv;
    }
    const S b4 = 4 * B2 * ir;
    q[1] = 0.5 * (fabs(p[1]) + sqrt(p[1] * p[1] + b4));
    q[2] = 0.5 * (fabs(p[2]) + sqrt(p[2] * p[2] + b4));
    q[3] = fabs(p[1]);
    q[4] = fabs(p[2]);
    const S isr = sqrt(ir);
    q[5] = p[5] * isr;
    q[6] = p[6] * isr;
    return;
  }
  if (first) q[0] = vv + eos_fast(P, p[0], p[4], B, B2);
  else q[0] = vv;
  q[1] = 0.5 * (fabs(p[1]) + sqrt(p[1] * p[1] + 4 * B2 / p[0]));
  q[2] = 0.5 * (fabs(p[2]) + sqrt(p[2] * p[2] + 4 * B2 / p[0]));
  q[3] = fabs(p[1]);
  q[4] = fabs(p[2]);
  q[5] = p[5] / sqrt(p[0]);
  q[6] = p[6] / sqrt(p[0]);
}
struct GlfMax {
  double v[kGlfQ];
};
__global__ void k_adj_argmax(DevParams P, const double* __restrict__ prim, GlfMax mx, int first,
                             unsigned long long* __restrict__ idx) {
  const long long N = P.N;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  double p[8], q[kGlfQ];
  load_cell<8>(prim, N, n, p);
  glf_quantities(P, p, first != 0, q);
  for (int s = 0; s < kGlfQ; ++s)
    if (q[s] == mx.v[s]) atomicMin(idx + s, (unsigned long long)n);
}
// lambda of each maximum -> its cell, through prim = con2pri(cons)
__global__ void k_adj_glf(DevParams P, const double* __restrict__ cons, const unsigned long long* __restrict__ idx,
                          const double* __restrict__ lam_s, int first, double* __restrict__ lam_cons) {
  const int s = threadIdx.x;
  if (s >= kGlfQ) return;
  const double ls = lam_s[s];
  const unsigned long long c = idx[s];
  if (ls == 0.0 || c >= (unsigned long long)P.N) return;
  const long long N = P.N;
  Dual<8> u[8], p[8], q[kGlfQ];
  for (int k = 0; k < 8; ++k) {
    u[k] = Dual<8>(cons[k * N + c]);
    u[k].d[k] = 1.0;
  }
  con2pri(P, p, u);
  glf_quantities(P, p, first != 0, q);
  for (int k = 0; k < 8; ++k) atomicAdd(lam_cons + k * N + c, ls * q[s].d[k]);
}

// ------------------------------------------------------------------ objective
// J = 1/2 |rho - rho_t|^2 + 1/2 |B - B_t|^2 over the cells; lambda = dJ/d cons
__global__ void k_adj_misfit(long long N, const double* __restrict__ cons, const double* __restrict__ rho_t,
                             const double* __restrict__ B_t, double* __restrict__ lam, double* __restrict__ J) {
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double s = 0.0;
  if (n < N) {
    for (int k = 0; k < 8; ++k) lam[k * N + n] = 0.0;
    const double d0 = cons[n] - rho_t[n];
    lam[n] = d0;
    s = 0.5 * d0 * d0;
    for (int k = 0; k < 3; ++k) {
      const double d = cons[(5 + k) * N + n] - B_t[k * N + n];
      lam[(5 + k) * N + n] = d;
      s += 0.5 * d * d;
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s != 0.0) atomicAdd(J, s);
}

// ------------------------------------------------------------------ host side
struct State {
  double* cons = nullptr;  // 8 planes, kept only for the final state
  double* prim = nullptr;  // 8 planes
  double* bx = nullptr;
  double* by = nullptr;
  double* A = nullptr;  // 3 planes
  DevScalars sc{};
};
struct StageSnap {
  double *Qe, *Qs, *bxQs, *byQs, *pe, *u1, *u2, *Fx, *Fy, *u3, *hh, *eta, *chit, *cf, *b1, *p1, *um, *b2, *p2;
  double* bct = nullptr;  // cell B after CT (Energy_Modify only)
  DevScalars sc;  // scalars of the stage (h, maxima)
  double mbig1, mbig2;
  bool second;
};

struct Adj {
  imex_ctx* ctx;
  size_t N;
  int R;
  double tol;
  std::vector<void*> mem;
  std::vector<StageSnap> snap;
  DevScalars step_sc{};  // scalars after the prologue of the recomputed step
  double* step_prim;     // prim at the start of the recomputed step
  // adjoint buffers
  double *lam_u, *lam_bx, *lam_by;                   // the running state adjoint (cons, faces)
  double *lam_cons_n, *lam_bx_n, *lam_by_n;          // adjoint at the step start
  double *lam_Hs, *lam_HsB;                          // stage derivatives
  double *l5, *l4, *lum, *l3, *l2, *l1;              // u_con after each sub-step (8 planes each)
  double *lbx5, *lby5, *lbxt, *lbyt, *lE, *lFx, *lFy;
  double *lQe, *lQs, *lbxQs, *lbyQs, *lpe, *lhh, *leta, *lchit, *lcf, *lrv, *lp, *mu, *w, *lw, *AT, *vdiag;
  double* lbsave = nullptr;  // adjoint of the cell B saved after the magnetic sub-system (Energy_Modify)
  double* dscal;  // device scalars: [0..4] GLF maxima adjoints, [5..6] magnetic cx cy (then the cA_x cA_y
                  // maxima adjoints), [7..8] pressure cvx cvy,
                  // [9] Mbig sum, [10] b min, [11] J
  unsigned long long* didx;  // argmax cells of the kGlfQ maxima, [7] argmin of b
  double* hscal;             // pinned mirror of dscal
};

imex_status amalloc(Adj& W, double** p, size_t count) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, (count ? count : 1) * sizeof(double));
  if (e != cudaSuccess) return cuda_check(W.ctx, e, "adjoint workspace");
  W.mem.push_back(q);
  *p = static_cast<double*>(q);
  return IMEX_OK;
}
void afree(Adj& W) {
  for (void* p : W.mem) cudaFree(p);
  W.mem.clear();
  if (W.hscal) cudaFreeHost(W.hscal);
  W.hscal = nullptr;
}
imex_status zero(Adj& W, double* p, size_t count) {
  return cuda_check(W.ctx, cudaMemsetAsync(p, 0, count * sizeof(double), W.ctx->stream), "adjoint clear");
}
imex_status copy(Adj& W, double* dst, const double* src, size_t count) {
  return cuda_check(W.ctx, cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyDeviceToDevice, W.ctx->stream),
                    "adjoint copy");
}
imex_status get_sc(imex_ctx* ctx, DevScalars* out) {
  cudaError_t e = cudaMemcpyAsync(ctx->h_sc, ctx->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) *out = *ctx->h_sc;
  return cuda_check(ctx, e, "adjoint scalars");
}
imex_status put_sc(imex_ctx* ctx, const DevScalars& in) {
  *ctx->h_sc = in;
  cudaError_t e = cudaMemcpyAsync(ctx->sc, ctx->h_sc, sizeof(DevScalars), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_check(ctx, e, "adjoint scalars");
}

imex_status workspace(Adj& W) {
  imex_ctx* ctx = W.ctx;
  const size_t N = W.N;
  imex_status s = IMEX_OK;
#define AL(p, c) \
  if (s == IMEX_OK) s = amalloc(W, &(p), (c))
  W.snap.resize(W.R);
  for (StageSnap& S : W.snap) {
    AL(S.Qe, 8 * N); AL(S.Qs, 8 * N); AL(S.bxQs, N); AL(S.byQs, N); AL(S.pe, N); AL(S.u1, 8 * N); AL(S.u2, 8 * N);
    AL(S.Fx, N); AL(S.Fy, N); AL(S.u3, 8 * N); AL(S.hh, N); AL(S.eta, N); AL(S.chit, N); AL(S.cf, N); AL(S.b1, N);
    AL(S.p1, N); AL(S.um, 8 * N); AL(S.b2, N); AL(S.p2, N);
    if (ctx->P.Energy_Modify) AL(S.bct, 3 * N);
  }
  AL(W.step_prim, 8 * N);
  AL(W.lam_u, 8 * N); AL(W.lam_bx, N); AL(W.lam_by, N);
  AL(W.lam_cons_n, 8 * N); AL(W.lam_bx_n, N); AL(W.lam_by_n, N);
  AL(W.lam_Hs, (size_t)W.R * 8 * N); AL(W.lam_HsB, (size_t)W.R * 2 * N);
  AL(W.l5, 8 * N); AL(W.l4, 8 * N); AL(W.lum, 8 * N); AL(W.l3, 8 * N); AL(W.l2, 8 * N); AL(W.l1, 8 * N);
  AL(W.lbx5, N); AL(W.lby5, N); AL(W.lbxt, N); AL(W.lbyt, N); AL(W.lE, N); AL(W.lFx, N); AL(W.lFy, N);
  AL(W.lQe, 8 * N); AL(W.lQs, 8 * N); AL(W.lbxQs, N); AL(W.lbyQs, N); AL(W.lpe, N); AL(W.lhh, N); AL(W.leta, N);
  AL(W.lchit, N); AL(W.lcf, N); AL(W.lrv, 3 * N); AL(W.lp, N); AL(W.mu, 3 * N); AL(W.w, 32 * N); AL(W.lw, 32 * N);
  AL(W.AT, 81 * N); AL(W.vdiag, N); AL(W.dscal, 16);
  if (ctx->P.Energy_Modify) AL(W.lbsave, 3 * N);
#undef AL
  if (s != IMEX_OK) return s;
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, 8 * sizeof(unsigned long long));
  if (e != cudaSuccess) return cuda_check(ctx, e, "adjoint workspace");
  W.mem.push_back(q);
  W.didx = static_cast<unsigned long long*>(q);
  e = cudaMallocHost(&q, 16 * sizeof(double));
  if (e != cudaSuccess) return cuda_check(ctx, e, "adjoint workspace");
  W.hscal = static_cast<double*>(q);
  return IMEX_OK;
}

imex_status save_state(Adj& W, State& st) {
  imex_ctx* ctx = W.ctx;
  const size_t N = W.N;
  imex_status s = IMEX_OK;
  if (!st.prim) {
    if ((s = amalloc(W, &st.prim, 8 * N)) != IMEX_OK || (s = amalloc(W, &st.bx, N)) != IMEX_OK ||
        (s = amalloc(W, &st.by, N)) != IMEX_OK || (s = amalloc(W, &st.A, 3 * N)) != IMEX_OK)
      return s;
  }
  if ((s = copy(W, st.prim, ctx->prim, 8 * N)) != IMEX_OK || (s = copy(W, st.bx, ctx->bx, N)) != IMEX_OK ||
      (s = copy(W, st.by, ctx->by, N)) != IMEX_OK || (s = copy(W, st.A, ctx->A, 3 * N)) != IMEX_OK)
    return s;
  return get_sc(ctx, &st.sc);
}
imex_status load_state(Adj& W, const State& st) {
  imex_ctx* ctx = W.ctx;
  const size_t N = W.N;
  imex_status s;
  if ((s = copy(W, ctx->prim, st.prim, 8 * N)) != IMEX_OK || (s = copy(W, ctx->bx, st.bx, N)) != IMEX_OK ||
      (s = copy(W, ctx->by, st.by, N)) != IMEX_OK || (s = copy(W, ctx->A, st.A, 3 * N)) != IMEX_OK)
    return s;
  return put_sc(ctx, st.sc);
}

// One step recomputed from the context's current state, keeping the sub-step states.
imex_status forward_step_snap(Adj& W) {
  imex_ctx* ctx = W.ctx;
  const size_t N = W.N;
  imex_status s;
  if ((s = copy(W, W.step_prim, ctx->prim, 8 * N)) != IMEX_OK) return s;
  if ((s = launch_step_prologue(ctx)) != IMEX_OK) return s;
  if ((s = get_sc(ctx, &W.step_sc)) != IMEX_OK) return s;
  for (int r = 0; r < W.R; ++r) {
    StageSnap& S = W.snap[r];
    if ((s = launch_stage_combine(ctx, r)) != IMEX_OK) return s;
    if ((s = get_sc(ctx, &S.sc)) != IMEX_OK) return s;
    copy(W, S.Qe, ctx->Qe, 8 * N);
    copy(W, S.Qs, ctx->Qs, 8 * N);
    copy(W, S.bxQs, ctx->bxQs, N);
    copy(W, S.byQs, ctx->byQs, N);
    copy(W, S.pe, ctx->pe, N);
    if ((s = launch_reconstruct(ctx, false)) != IMEX_OK || (s = launch_flux_update(ctx, 0)) != IMEX_OK) return s;
    copy(W, S.u1, ctx->cons, 8 * N);
    if ((s = mag_rhs(ctx)) != IMEX_OK) return s;
    int op;
    double* x;
    const double* b;
    mag_system(ctx, &op, &x, &b);
    if ((s = run_gmres(ctx, op, x, b)) != IMEX_OK) return s;
    copy(W, S.u2, ctx->cons, 8 * N);
    if ((s = mag_out(ctx)) != IMEX_OK) return s;
    if (ctx->P.Energy_Modify) copy(W, ctx->Bsave, ctx->cons + 5 * N, 3 * N);  // as run_stage does
    copy(W, S.Fx, ctx->Fx, N);
    copy(W, S.Fy, ctx->Fy, N);
    if ((s = launch_flux_update(ctx, 1)) != IMEX_OK) return s;
    copy(W, S.u3, ctx->cons, 8 * N);
    if ((s = pres_part1(ctx)) != IMEX_OK) return s;
    copy(W, S.hh, ctx->hh, N);
    copy(W, S.eta, ctx->eta, N);
    copy(W, S.chit, ctx->chit, N);
    copy(W, S.b1, ctx->pb, N);
    if ((s = run_nested_newton(ctx, ctx->pp, ctx->pb)) != IMEX_OK) return s;
    copy(W, S.p1, ctx->pp, N);
    DevScalars t;
    if ((s = get_sc(ctx, &t)) != IMEX_OK) return s;
    S.mbig1 = t.Mbig;
    if ((s = pres_part2(ctx, r, &S.second)) != IMEX_OK) return s;
    copy(W, S.um, ctx->cons, 8 * N);
    copy(W, S.b2, ctx->pb, N);
    if (S.second) {
      if ((s = run_nested_newton(ctx, ctx->pp, ctx->pb)) != IMEX_OK) return s;
      copy(W, S.p2, ctx->pp, N);
      if ((s = get_sc(ctx, &t)) != IMEX_OK) return s;
      S.mbig2 = t.Mbig;
    }
    if ((s = pres_part3(ctx)) != IMEX_OK) return s;
    if ((s = launch_ct(ctx, 0)) != IMEX_OK) return s;
    if (ctx->P.Energy_Modify) copy(W, S.bct, ctx->cons + 5 * N, 3 * N);
    if ((s = launch_stage_derivative(ctx, r)) != IMEX_OK) return s;
  }
  return imex_end_step(ctx);
}

// cf of the shock detector for the adjoint (recomputed: the forward keeps only chi~ and eta)
__global__ void k_adj_cf(DevParams P, const double* __restrict__ Q, double* __restrict__ cf) {
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= P.N) return;
  double c[8];
  load_cell<8>(Q, P.N, n, c);
  double p = pressure_of(P, c);
  double a2 = eos_a2(P, c[0], p);
  double cA2 = (c[5] * c[5] + c[6] * c[6] + c[7] * c[7]) / c[0];
  cf[n] = sqrt(a2 + cA2);
}

// adjoint of one nested-Newton (or linear) pressure solve at its solution p, right-hand
// side b, slope Mbig: mu = J^{-T} lam_p, lam_b += mu (into lb), lam_hh/eta/cv -= mu^T dg/dtheta
imex_status newton_adjoint(Adj& W, const StageSnap& S, const double* p, const double* b, double mbig,
                           const double* lam_p, double* mu_out) {
  imex_ctx* ctx = W.ctx;
  const DevParams& P = ctx->P;
  const size_t N = W.N;
  const bool newton = P.floor_on || P.eos_type != IMEX_IDEAL_GAS;
  AdjOp a{};
  a.kind = newton ? ADJ_OP_PRESSURE_J : ADJ_OP_PRESSURE_L;
  a.hh = S.hh;
  a.eta = S.eta;
  a.rho = S.u3;  // u_con density during the pressure sub-system
  a.vscale = ctx->vscale;
  a.vdiag = W.vdiag;
  imex_status s;
  if (newton) {
    k_adj_vdiag<<<ablocks(N), kAT, 0, ctx->stream>>>(P, mbig, p, S.u3, W.vdiag);
    ACHECK(ctx, "k_adj_vdiag");
  }
  if ((s = adj_transpose_solve(ctx, a, W.AT, mu_out, lam_p, W.tol)) != IMEX_OK) return s;
  // the residual's dependence on the frozen coefficients is that of the L-mode operator at p
  AdjOp l = a;
  l.kind = ADJ_OP_PRESSURE_L;
  double* lq[4] = {W.lhh, W.leta, nullptr, nullptr};
  if ((s = adj_coef_vjp(ctx, l, p, mu_out, lq, W.dscal + 7)) != IMEX_OK) return s;
  if (P.floor_on) {
    // Cor.1: g depends on Mbig in floored cells, and Mbig = max(M_base, M_cor(min b))
    W.hscal[0] = 0.0;
    cudaMemcpyAsync(W.dscal + 9, W.hscal, sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
    k_adj_mbig_sum<<<ablocks(N), kAT, 0, ctx->stream>>>(P, p, mu_out, W.dscal + 9);
    W.hscal[1] = INFINITY;
    cudaMemcpyAsync(W.dscal + 10, W.hscal + 1, sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
    k_min_reduce<<<64, kAT, 0, ctx->stream>>>((long long)N, b, W.dscal + 10);
    ACHECK(ctx, "adjoint Mbig");
    cudaError_t e = cudaMemcpyAsync(W.hscal + 2, W.dscal + 9, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_check(ctx, e, "adjoint Mbig");
    const double lam_mbig = -W.hscal[2], bmin = W.hscal[3];
    const double Vpe = P.p_floor / (P.gamma - 1.0);
    const double M_cor = (Vpe - bmin > 0.0 ? Vpe - bmin : 0.0) / ((1.0 - P.theta) * P.p_floor);
    const double M_base = P.Mbig_fac / (P.gamma - 1.0);
    if (lam_mbig != 0.0 && M_cor > M_base && Vpe - bmin > 0.0) {
      unsigned long long big = ~0ull;
      cudaMemcpyAsync(W.didx + 7, &big, sizeof(big), cudaMemcpyHostToDevice, ctx->stream);
      k_adj_bmin<<<ablocks(N), kAT, 0, ctx->stream>>>((long long)N, b, bmin, W.didx + 7);
      unsigned long long at = 0;
      e = cudaMemcpyAsync(&at, W.didx + 7, sizeof(at), cudaMemcpyDeviceToHost, ctx->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
      if (e != cudaSuccess) return cuda_check(ctx, e, "adjoint Mbig");
      if (at < N) {
        // mu (= lam_b) at the argmin gains lam_Mbig dMbig/db_min
        W.hscal[4] = lam_mbig * (-1.0 / ((1.0 - P.theta) * P.p_floor));
        e = cudaMemcpyAsync(W.dscal + 12, W.hscal + 4, sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return cuda_check(ctx, e, "adjoint Mbig");
        k_axpy_planes<<<1, 1, 0, ctx->stream>>>(1, mu_out + at, W.dscal + 12, 1.0);
        ACHECK(ctx, "adjoint Mbig");
      }
    }
  }
  return IMEX_OK;
}

// The adjoint of one recomputed step: lam_u, lam_bx, lam_by (of the step's end state) become
// the adjoint of its start state (cons at the step start, faces).
imex_status reverse_step(Adj& W) {
  imex_ctx* ctx = W.ctx;
  const DevParams& P = ctx->P;
  const size_t N = W.N;
  const int nb = ablocks(N);
  cudaStream_t st = ctx->stream;
  imex_status s;
  double ae[kMaxRK][kMaxRK], ai[kMaxRK][kMaxRK];
  tableau(W.R, ae, ai);
  zero(W, W.lam_Hs, (size_t)W.R * 8 * N);
  zero(W, W.lam_HsB, (size_t)W.R * 2 * N);
  zero(W, W.lam_cons_n, 8 * N);
  zero(W, W.lam_bx_n, N);
  zero(W, W.lam_by_n, N);
  zero(W, W.dscal, 16);
  const double dt = W.step_sc.dt;
  for (int r = W.R - 1; r >= 0; --r) {
    const StageSnap& S = W.snap[r];
    if ((s = put_sc(ctx, S.sc)) != IMEX_OK) return s;
    const double h = S.sc.h, adt = S.sc.adt;
    const bool last = r == W.R - 1;
    // (1) stage derivative
    prof_begin(ctx);
    k_adj_derivative<<<nb, kAT, 0, st>>>(P, r, adt, last ? W.lam_u : nullptr, last ? W.lam_bx : nullptr,
                                          last ? W.lam_by : nullptr, W.lam_Hs, W.lam_HsB, W.l5, W.lQs, W.lbx5, W.lby5,
                                          W.lbxQs, W.lbyQs, S.bct, S.u2 + 5 * N, W.lbsave);
    // (2) CT faces and cell B
    k_adj_ct_faces1<<<nb, kAT, 0, st>>>(P, W.l5, W.lbx5, W.lby5, W.lbxt, W.lbyt, W.lbxQs, W.lbyQs, W.l4);
    k_adj_ct_faces2<<<nb, kAT, 0, st>>>(P, h, W.lbxt, W.lbyt, W.lE);
    ACHECK(ctx, "adjoint CT faces");
    prof_end(ctx, F_ADJ_LINEAR, 0.0, 3);
    // (3) CT corner EMF: inputs Fx, Fy, u_con after the pressure sub-system (= um with E of p)
    // u4 is not kept: its planes other than E equal um, and the corner reads none of E
    zero(W, W.lFx, N);
    zero(W, W.lFy, N);
    {
      CellVjp A = cv_empty();
      const unsigned cN = 1u << NB_N, cE = 1u << NB_E, cNE = 1u << NB_NE;
      cv_arr(A, CC_FX, S.Fx, W.lFx, 0, 1, OFS_C | cN);
      cv_arr(A, CC_FY, S.Fy, W.lFy, 0, 1, OFS_C | cE);
      cv_arr_planes(A, CC_UCON, S.um, W.l4, 0x67u, OFS_C | cE | cN | cNE);  // rho, mx, my, Bx, By
      A.lam_out[0] = W.lE;
      A.sx = -1.0;
      A.sy = 1.0;
      if ((s = run_cell_vjp<4>(ctx, A, FnCtCorner{})) != IMEX_OK) return s;
    }
    // (4) pressure sub-system
    zero(W, W.lum, 8 * N);
    zero(W, W.lp, N);
    zero(W, W.lhh, N);
    zero(W, W.leta, N);
    zero(W, W.lrv, 3 * N);
    zero(W, W.l3, 8 * N);
    zero(W, W.lQe, 8 * N);
    zero(W, W.lpe, N);
    const double* pE = S.second ? S.p2 : S.p1;
    if (P.U_update == IMEX_ConservationofU) {
      // E -= h div(h_e rho v) at the final pressure, on um (its E plane is the old energy)
      CellVjp A = cv_empty();
      cv_arr(A, EC_P, pE, W.lp, 0, 1, OFS_CROSS);
      cv_arr_planes(A, EC_UCON, S.um, W.lum, 0x17u, OFS_CROSS);  // rho, mx, my, E
      A.lam_out[0] = W.l4 + 4 * N;
      A.h = h;
      if ((s = run_cell_vjp<4>(ctx, A, FnEnergyCons{})) != IMEX_OK) return s;
    } else {  // DefinitionofU at the final pressure, on um
      CellVjp A = cv_empty();
      cv_arr(A, ED_P, pE, W.lp, 0, 1, OFS_C);
      cv_arr(A, ED_UCON, S.um, W.lum, 0, 8, OFS_C);
      A.lam_out[0] = W.l4 + 4 * N;
      if ((s = run_cell_vjp<4>(ctx, A, FnEnergyDef{})) != IMEX_OK) return s;
    }
    // passthrough of the planes other than E
    for (int k = 0; k < 8; ++k)
      if (k != 4) k_axpy_planes<<<ablocks(N), kAT, 0, st>>>((long long)N, W.lum + k * N, W.l4 + k * N, 1.0);
    if (S.second) {
      if ((s = newton_adjoint(W, S, S.p2, S.b2, S.mbig2, W.lp, W.mu)) != IMEX_OK) return s;
      CellVjp A = cv_empty();  // b2 = rhs(um, hh, rv, kin = um momentum)
      cv_arr(A, PR_UCON, S.um, W.lum, 0, 8, OFS_C);
      cv_arr(A, PR_HH, S.hh, W.lhh, 0, 1, OFS_CROSS);
      cv_arr(A, PR_RV, S.u3 + N, W.lrv, 0, 2, OFS_CROSS);
      cv_arr(A, PR_KIN, S.um + N, W.lum + N, 0, 3, OFS_C);
      A.lam_out[0] = W.mu;
      A.h = h;
      if ((s = run_cell_vjp<4>(ctx, A, FnPresRhs{})) != IMEX_OK) return s;
      zero(W, W.lp, N);
    }
    {  // momentum: um[1..2] = rv - h grad p1
      CellVjp A = cv_empty();
      cv_arr(A, MO_P, S.p1, W.lp, 0, 1, OFS_CROSS);
      cv_arr(A, MO_RV, S.u3 + N, W.lrv, 0, 2, OFS_C);
      A.lam_out[0] = W.lum + N;
      A.lam_out[1] = W.lum + 2 * N;
      A.h = h;
      if ((s = run_cell_vjp<4>(ctx, A, FnMomentum{})) != IMEX_OK) return s;
    }
    // um = u3 except momentum x, y
    for (int k = 0; k < 8; ++k)
      if (k != 1 && k != 2) k_axpy_planes<<<ablocks(N), kAT, 0, st>>>((long long)N, W.l3 + k * N, W.lum + k * N, 1.0);
    if (!S.second) {
      // without a second solve the energy used p1: its adjoint is already in lp
    }
    if ((s = newton_adjoint(W, S, S.p1, S.b1, S.mbig1, W.lp, W.mu)) != IMEX_OK) return s;
    {  // b1 = rhs(u3, hh, rv, kin = rv)
      CellVjp A = cv_empty();
      cv_arr(A, PR_UCON, S.u3, W.l3, 0, 8, OFS_C);
      cv_arr(A, PR_HH, S.hh, W.lhh, 0, 1, OFS_CROSS);
      cv_arr(A, PR_RV, S.u3 + N, W.lrv, 0, 2, OFS_CROSS);
      cv_arr(A, PR_KIN, S.u3 + N, W.lrv, 0, 3, OFS_C);
      A.lam_out[0] = W.mu;
      A.h = h;
      if ((s = run_cell_vjp<4>(ctx, A, FnPresRhs{})) != IMEX_OK) return s;
    }
    k_axpy_planes<<<ablocks(3 * N), kAT, 0, st>>>((long long)(3 * N), W.l3 + N, W.lrv, 1.0);
    {  // hh = h(Qe) rho_e / rho
      CellVjp A = cv_empty();
      cv_arr(A, HH_QE, S.Qe, W.lQe, 0, 8, OFS_C);
      cv_arr(A, HH_UCON, S.u3, W.l3, 0, 1, OFS_C);
      A.lam_out[0] = W.lhh;
      if ((s = run_cell_vjp<4>(ctx, A, FnHh{})) != IMEX_OK) return s;
    }
    // shock detector eta(Qe)
    zero(W, W.lchit, N);
    zero(W, W.lcf, N);
    k_adj_cf<<<nb, kAT, 0, st>>>(P, S.Qe, W.vdiag);  // cf into scratch
    k_adj_shock_max<<<nb, kAT, 0, st>>>(P, S.chit, W.leta, W.lchit);
    k_adj_shock_tilde<<<nb, kAT, 0, st>>>(P, S.Qe, W.vdiag, W.lchit, W.lQe, W.lcf);
    ACHECK(ctx, "adjoint shock detector");
    {
      CellVjp A = cv_empty();
      cv_arr(A, 0, S.Qe, W.lQe, 0, 8, OFS_C);
      A.lam_out[0] = W.lcf;
      if ((s = run_cell_vjp<4>(ctx, A, FnShockCf{})) != IMEX_OK) return s;
    }
    // (5) pressure-form flux: u3[0..4] = Qs - h div F(w(Qe), B of u2, a_max)
    zero(W, W.l2, 8 * N);
    zero(W, W.lw, 32 * N);
    if ((s = copy(W, ctx->Qe, S.Qe, 8 * N)) != IMEX_OK) return s;
    if ((s = launch_reconstruct(ctx, false)) != IMEX_OK) return s;
    if ((s = copy(W, W.w, ctx->w, 32 * N)) != IMEX_OK) return s;
    prof_begin(ctx);
    k_adj_flux<1><<<nb, kAT, 0, st>>>(P, h, S.sc.a_max, W.w, S.u2, W.l3, W.lw, W.l2, W.lQs, W.dscal + 0);
    adj_recon(P, st, S.Qe, W.lw, W.lQe);
    ACHECK(ctx, "adjoint pressure flux");
    prof_end(ctx, F_ADJ_FLUX, 0.0, 2);
    for (int k = 5; k < 8; ++k) k_axpy_planes<<<ablocks(N), kAT, 0, st>>>((long long)N, W.l2 + k * N, W.l3 + k * N, 1.0);
    if (P.Energy_Modify)  // the saved B is the B of u2
      k_axpy_planes<<<ablocks(3 * N), kAT, 0, st>>>((long long)(3 * N), W.l2 + 5 * N, W.lbsave, 1.0);
    // (6) CollectMagFluxes
    {
      CellVjp A = cv_empty();
      cv_arr_planes(A, CF_UCON, S.u2, W.l2, 0xE7u, OFS_NO_SW);  // rho, mx, my, B
      cv_arr(A, CF_QE, S.Qe, W.lQe, 5, 3, OFS_NO_SW);
      cv_arr(A, CF_PE, S.pe, W.lpe, 0, 1, OFS_NO_SW);
      A.lam_out[0] = W.lFx;
      A.lam_out[1] = W.lFy;
      A.sval[0] = S.sc.B_max_x;
      A.sval[1] = S.sc.B_max_y;
      A.lam_s = W.dscal + 1;
      A.h = h;
      if ((s = run_cell_vjp<4>(ctx, A, FnCollect{})) != IMEX_OK) return s;
    }
    // (7) magnetic solve A(Qe B, rho) x = b with x = B of u2
    {
      AdjOp a{};
      a.kind = ADJ_OP_MAGNETIC_B;
      a.Qe = S.Qe;
      a.rho = S.u1;
      if ((s = adj_transpose_solve(ctx, a, W.AT, W.mu, W.l2 + 5 * N, W.tol)) != IMEX_OK) return s;
      zero(W, W.l1, 8 * N);
      double* lq[4] = {W.lQe + 5 * N, W.lQe + 6 * N, W.lQe + 7 * N, W.l1};
      if ((s = adj_coef_vjp(ctx, a, S.u2 + 5 * N, W.mu, lq, W.dscal + 5)) != IMEX_OK) return s;
    }
    for (int k = 0; k < 5; ++k) k_axpy_planes<<<ablocks(N), kAT, 0, st>>>((long long)N, W.l1 + k * N, W.l2 + k * N, 1.0);
    // (8) magnetic right-hand side b(u1, Qe, pe, Qs)
    {
      CellVjp A = cv_empty();
      cv_arr(A, MR_UCON, S.u1, W.l1, 0, 4, OFS_CROSS);
      cv_arr(A, MR_QE, S.Qe, W.lQe, 5, 3, OFS_CROSS);
      cv_arr(A, MR_PE, S.pe, W.lpe, 0, 1, OFS_ALL);
      cv_arr(A, MR_QS, S.Qs, nullptr, 0, 0, OFS_C);
      A.lam_out[0] = W.mu;
      A.lam_out[1] = W.mu + N;
      A.lam_out[2] = W.mu + 2 * N;
      A.h = h;
      if ((s = run_cell_vjp<4>(ctx, A, FnMagRhs{})) != IMEX_OK) return s;
    }
    k_axpy_planes<<<ablocks(3 * N), kAT, 0, st>>>((long long)(3 * N), W.lQs + 5 * N, W.mu, 1.0);
    // (9) convective flux: u1[0..4] = Qs - h div F(w(Qe), a_max)
    zero(W, W.lw, 32 * N);
    prof_begin(ctx);
    k_adj_flux<0><<<nb, kAT, 0, st>>>(P, h, S.sc.a_max, W.w, S.u1, W.l1, W.lw, nullptr, W.lQs, W.dscal + 0);
    adj_recon(P, st, S.Qe, W.lw, W.lQe);
    ACHECK(ctx, "adjoint convective flux");
    prof_end(ctx, F_ADJ_FLUX, 0.0, 2);
    // (10) p(Qe) of the combination
    {
      CellVjp A = cv_empty();
      cv_arr(A, 0, S.Qe, W.lQe, 0, 8, OFS_C);
      A.lam_out[0] = W.lpe;
      if ((s = run_cell_vjp<4>(ctx, A, FnPe{})) != IMEX_OK) return s;
    }
    // (11) stage combination
    Coefs T{};
    for (int q = 0; q < kMaxRK; ++q) {
      T.ae[q] = ae[r][q];
      T.ai[q] = ai[r][q];
    }
    k_adj_combine<<<nb, kAT, 0, st>>>(P, T, r, dt, W.lQe, W.lQs, W.lbxQs, W.lbyQs, W.lam_cons_n, W.lam_Hs, W.lam_bx_n,
                                       W.lam_by_n, W.lam_HsB);
    ACHECK(ctx, "adjoint combination");
    ctx->kernel_launches += 20;  // the linear helpers (axpy, shock, combine) outside the profiled families
  }
  // GLF maxima of the step prologue, from prim = con2pri(cons_n)
  {
    // viscosity scalars -> maxima: cx = B_max_x dx / dx^2, cvx = vx_max dx / dx^2 (MaterialSpeedp)
    cudaError_t e = cudaMemcpyAsync(W.hscal, W.dscal, 9 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_check(ctx, e, "adjoint maxima");
    W.hscal[1] += W.hscal[5] * (P.dx / (P.dx * P.dx));
    W.hscal[2] += W.hscal[6] * (P.dy / (P.dy * P.dy));
    if (P.add_pvisc == IMEX_MaterialSpeedp) {
      W.hscal[3] += W.hscal[7] * (P.dx / (P.dx * P.dx));
      W.hscal[4] += W.hscal[8] * (P.dy / (P.dy * P.dy));
    }
    // slots 5 and 6 (the magnetic viscosity's, taken into 1 and 2 above) now carry cA_x, cA_y
    W.hscal[5] = W.hscal[6] = 0.0;
    if (P.add_pvisc == IMEX_AlfvenSpeedp) {  // cvx = cA_x dx / dx^2
      W.hscal[5] = W.hscal[7] * (P.dx / (P.dx * P.dx));
      W.hscal[6] = W.hscal[8] * (P.dy / (P.dy * P.dy));
    }
    e = cudaMemcpyAsync(W.dscal, W.hscal, kGlfQ * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_check(ctx, e, "adjoint maxima");
    const bool first = W.step_sc.timestep <= 1;
    GlfMax mx{};
    mx.v[0] = first ? W.step_sc.ch : W.step_sc.v_max;
    mx.v[1] = W.step_sc.B_max_x;
    mx.v[2] = W.step_sc.B_max_y;
    mx.v[3] = W.step_sc.vx_max;
    mx.v[4] = W.step_sc.vy_max;
    mx.v[5] = W.step_sc.cA_x;
    mx.v[6] = W.step_sc.cA_y;
    e = cudaMemsetAsync(W.didx, 0xff, kGlfQ * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return cuda_check(ctx, e, "adjoint maxima");
    k_adj_argmax<<<nb, kAT, 0, st>>>(P, W.step_prim, mx, first ? 1 : 0, W.didx);
    // cons at the step start = pri2con(prim) (cons_n of the prologue)
    k_adj_glf<<<1, 32, 0, st>>>(P, ctx->cons_n, W.didx, W.dscal, first ? 1 : 0, W.lam_cons_n);
    ACHECK(ctx, "adjoint maxima");
  }
  if ((s = copy(W, W.lam_u, W.lam_cons_n, 8 * N)) != IMEX_OK) return s;
  if ((s = copy(W, W.lam_bx, W.lam_bx_n, N)) != IMEX_OK) return s;
  return copy(W, W.lam_by, W.lam_by_n, N);
}

imex_status supported(imex_ctx* ctx) {
  const DevParams& P = ctx->P;
  const char* why = nullptr;
  if (P.formula != IMEX_PressureFormula) why = "the pressure formula";
  else if (P.magfield != IMEX_StaggerCT) why = "StaggerCT";
  else if (P.eos_type != IMEX_IDEAL_GAS) why = "the ideal-gas EOS";
  else if (!P.GLF) why = "GLF";
  else if (!(P.fixed_dt > 0.0)) why = "a fixed time step (fixed_dt > 0)";
  else if (ctx->cfg.precision != IMEX_PRECISION_FP64) why = "FP64 precision";
  else if (P.xclamp || P.yclamp) why = "periodic boundaries";
  if (!why) return IMEX_OK;
  return set_error(ctx, IMEX_ERR_UNSUPPORTED, std::string("the adjoint needs ") + why);
}

// forward nsteps with checkpoints, cotangent from `seed` at the final state, reverse sweep;
// gradients w.r.t. the initial primitive planes and face fields
imex_status adjoint_core(imex_ctx* ctx, const imex_adjoint_opts* o, const std::function<imex_status(Adj&)>& seed,
                         double* g_prim, double* g_bx, double* g_by) {
  imex_status s = supported(ctx);
  if (s != IMEX_OK) return s;
  if (!o || o->nsteps < 1 || o->checkpoint_every < 1) return set_error(ctx, IMEX_ERR_INVALID, "bad adjoint options");
  Adj W{};
  W.ctx = ctx;
  W.N = ctx->N;
  // the forward recomputations keep the shock detector's chi~ (its VJP follows the branches)
  struct KeepChit {
    imex_ctx* c;
    ~KeepChit() { c->keep_shock_chit = false; }
  } keep{ctx};
  ctx->keep_shock_chit = true;
  W.R = ctx->P.RKs;
  W.tol = o->gmres_tol > 0.0 ? o->gmres_tol : 1e-13;
  const size_t N = W.N;
  auto run = [&]() -> imex_status {
    imex_status t = workspace(W);
    if (t != IMEX_OK) return t;
    const int K = o->checkpoint_every, nsteps = o->nsteps;
    const int nseg = (nsteps + K - 1) / K;
    std::vector<State> ck(nseg), seg(K);
    State start{}, fin{};
    if ((t = save_state(W, start)) != IMEX_OK) return t;
    for (int st = 0; st < nsteps; ++st) {
      if (st % K == 0 && (t = save_state(W, ck[st / K])) != IMEX_OK) return t;
      if ((t = imex_step(ctx, nullptr)) != IMEX_OK) return t;
    }
    if ((t = save_state(W, fin)) != IMEX_OK) return t;
    if ((t = amalloc(W, &fin.cons, 8 * N)) != IMEX_OK || (t = copy(W, fin.cons, ctx->cons, 8 * N)) != IMEX_OK) return t;
    // cotangent of the final state (cons, faces)
    zero(W, W.lam_bx, N);
    zero(W, W.lam_by, N);
    if ((t = seed(W)) != IMEX_OK) return t;
    for (int g = nseg - 1; g >= 0; --g) {
      const int s0 = g * K, s1 = (s0 + K < nsteps) ? s0 + K : nsteps;
      if ((t = load_state(W, ck[g])) != IMEX_OK) return t;
      for (int st = s0; st < s1; ++st) {
        if ((t = save_state(W, seg[st - s0])) != IMEX_OK) return t;
        if (st + 1 < s1 && (t = imex_step(ctx, nullptr)) != IMEX_OK) return t;
      }
      for (int st = s1 - 1; st >= s0; --st) {
        if ((t = load_state(W, seg[st - s0])) != IMEX_OK) return t;
        if ((t = forward_step_snap(W)) != IMEX_OK) return t;
        if ((t = reverse_step(W)) != IMEX_OK) return t;
      }
    }
    // prim at t = 0 -> cons = pri2con(prim) of the first step
    if (g_prim) {
      double* gp;
      if ((t = amalloc(W, &gp, 8 * N)) != IMEX_OK || (t = zero(W, gp, 8 * N)) != IMEX_OK) return t;
      CellVjp A = cv_empty();
      cv_arr(A, 0, start.prim, gp, 0, 8, OFS_C);
      for (int k = 0; k < 8; ++k) A.lam_out[k] = W.lam_u + k * N;
      if ((t = run_cell_vjp<4>(ctx, A, FnPri2Con{})) != IMEX_OK) return t;
      cudaError_t e = cudaMemcpyAsync(g_prim, gp, 8 * N * sizeof(double), cudaMemcpyDefault, ctx->stream);
      if (e != cudaSuccess) return cuda_check(ctx, e, "gradient download");
    }
    cudaError_t e = cudaSuccess;
    if (g_bx) e = cudaMemcpyAsync(g_bx, W.lam_bx, N * sizeof(double), cudaMemcpyDefault, ctx->stream);
    if (g_by && e == cudaSuccess) e = cudaMemcpyAsync(g_by, W.lam_by, N * sizeof(double), cudaMemcpyDefault, ctx->stream);
    if (e != cudaSuccess) return cuda_check(ctx, e, "gradient download");
    // leave the context at the final state of the forward run
    if ((t = load_state(W, fin)) != IMEX_OK) return t;
    if ((t = copy(W, ctx->cons, fin.cons, 8 * N)) != IMEX_OK) return t;
    return cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "adjoint");
  };
  s = run();
  cudaStreamSynchronize(ctx->stream);
  afree(W);
  return s;
}

}  // namespace
}  // namespace imex

using namespace imex;

extern "C" {

imex_status imex_adjoint_run(imex_ctx* ctx, const imex_adjoint_opts* opts, const double* rho_target,
                             const double* B_target, double* J, double* g_prim, double* g_bx, double* g_by) {
  if (!ctx || !opts || !rho_target || !B_target) return IMEX_ERR_INVALID;
  double* dt_rho = nullptr;
  double* dt_B = nullptr;
  auto seed = [&](Adj& W) -> imex_status {
    imex_ctx* c = W.ctx;
    const size_t N = W.N;
    imex_status t;
    if ((t = amalloc(W, &dt_rho, N)) != IMEX_OK || (t = amalloc(W, &dt_B, 3 * N)) != IMEX_OK) return t;
    cudaError_t e = cudaMemcpyAsync(dt_rho, rho_target, N * sizeof(double), cudaMemcpyDefault, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt_B, B_target, 3 * N * sizeof(double), cudaMemcpyDefault, c->stream);
    if (e != cudaSuccess) return cuda_check(c, e, "target upload");
    zero(W, W.dscal + 11, 1);
    k_adj_misfit<<<ablocks(N), kAT, 0, c->stream>>>((long long)N, c->cons, dt_rho, dt_B, W.lam_u, W.dscal + 11);
    ACHECK(c, "k_adj_misfit");
    if (J) {
      e = cudaMemcpyAsync(W.hscal + 11, W.dscal + 11, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
      if (e != cudaSuccess) return cuda_check(c, e, "misfit");
      *J = W.hscal[11];
    }
    return IMEX_OK;
  };
  return adjoint_core(ctx, opts, seed, g_prim, g_bx, g_by);
}

imex_status imex_adjoint_vjp(imex_ctx* ctx, const imex_adjoint_opts* opts, const double* lam_cons,
                             const double* lam_bx, const double* lam_by, double* g_prim, double* g_bx, double* g_by) {
  if (!ctx || !opts || !lam_cons) return IMEX_ERR_INVALID;
  auto seed = [&](Adj& W) -> imex_status {
    imex_ctx* c = W.ctx;
    const size_t N = W.N;
    cudaError_t e = cudaMemcpyAsync(W.lam_u, lam_cons, 8 * N * sizeof(double), cudaMemcpyDefault, c->stream);
    if (lam_bx && e == cudaSuccess) e = cudaMemcpyAsync(W.lam_bx, lam_bx, N * sizeof(double), cudaMemcpyDefault, c->stream);
    if (lam_by && e == cudaSuccess) e = cudaMemcpyAsync(W.lam_by, lam_by, N * sizeof(double), cudaMemcpyDefault, c->stream);
    return cuda_check(c, e, "cotangent upload");
  };
  return adjoint_core(ctx, opts, seed, g_prim, g_bx, g_by);
}

}  // extern "C"
