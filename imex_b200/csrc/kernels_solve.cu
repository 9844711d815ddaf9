// Implicit sub-systems of one IMEX stage: matrix-free operators, restarted
// GMRES as one persistent cooperative kernel, the nested-Newton pressure
// solve, and the surrounding right-hand-side / update kernels.
//
// GMRES(k) (implicit_operators.cpp:793-919): classical Gram-Schmidt, Givens
// rotations, left preconditioning, tolerance GMREStol*|r0| + GMREStol.
// Device layout of one Arnoldi step j, done as ONE pass over the grid plus
// ONE grid barrier:
//   each CTA, per 32x16 tile: w = Av_j - sum_i H[i][j] v_i on the tile plus a
//   halo (shared memory), w -> basis slot j+1 (unnormalised), Aw = M^-1 A w on
//   the tile from shared memory, and partial sums of v_i.Aw, w.Aw, w.w;
//   barrier; every CTA reduces the partials in the same fixed order, so all
//   CTAs hold identical Hessenberg columns and take identical branches.
// Basis vectors are never rescaled in memory: v_i = sigma_i * V_i with
// sigma_i = 1/|w_{i-1}| kept in shared memory.
#include <cooperative_groups.h>

#include <algorithm>
#include <type_traits>
#include <cstdio>
#include <cstring>
#include <functional>
#include <vector>

#include "cells.cuh"
#include "launch.cuh"

namespace imex {
namespace {

constexpr int TX = 32, TY = 16, NT = 256;
constexpr int KCAP = 30;        // largest supported restart length
constexpr int NP = KCAP + 2;    // partial-sum slots per CTA

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
// Krylov vectors are stored as double (plain form) or float (mixed form); both load as double
__device__ __forceinline__ double ldv(const double* p) { return __ldcg(p); }
__device__ __forceinline__ double ldv(const float* p) { return (double)__ldcg(p); }

// ------------------------------------------------------------------ grid barrier
// Bounded barrier over a cooperative launch (all CTAs co-resident).  The arrival
// counter only ever grows: barrier number g is complete once it reaches
// (g + 1) * nblk, so the last CTA to arrive releases everyone with its own
// arrival (no reset, no second counter).  The counter is 64-bit, so it cannot wrap
// within a launch (a 32-bit one would after 2^32 / nblk barriers, and the target
// computed from a wrapped count would be wrong when nblk is not a power of two).
// Arrival is a release atomic and the wait ends with an acquire fence, so the
// CTA's writes before the barrier are visible to every CTA after it.  The wait
// polls with relaxed loads: an acquire load per poll would invalidate the SM's L1
// on every poll, under the feet of the other CTA working on the same SM.  A wait
// longer than s->wait_cycles SM cycles sets the abort flag; every CTA then
// returns false and the caller leaves the kernel.
__device__ __forceinline__ unsigned long long ld_relaxed_gpu(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ unsigned long long atom_add_release_gpu(unsigned long long* p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.release.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}
__device__ bool grid_barrier(SyncState* s, unsigned nblk) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    const unsigned long long old = atom_add_release_gpu(&s->count, 1ull);
    const unsigned long long target = (old / nblk + 1ull) * nblk;
    const long long limit = s->wait_cycles;
    const long long t0 = clock64();
    for (unsigned spin = 0;; ++spin) {
      if (ld_relaxed_gpu(&s->count) >= target) break;
      __nanosleep(32);
      if ((spin & 15u) == 15u) {
        if (*((volatile int*)&s->abort)) {
          ok = 0;
          break;
        }
        if (clock64() - t0 > limit) {
          atomicExch(&s->abort, 1);
          ok = 0;
          break;
        }
      }
    }
    fence_acq_rel_gpu();
  }
  __syncthreads();
  return ok != 0;
}

// ------------------------------------------------------------------ tiling
struct Tiling {
  int nx, ny, tiles_x, ntiles;
  long long N;
  int xclamp, yclamp;  // transmissive directions: the halo clamps instead of wrapping
};
// tiles of tx x ty cells (the operator's tile shape, TileShape below)
__host__ __device__ inline Tiling make_tiling(int nx, int ny, int xclamp = 0, int yclamp = 0, int tx = TX, int ty = TY) {
  Tiling t;
  t.nx = nx;
  t.ny = ny;
  t.xclamp = xclamp;
  t.yclamp = yclamp;
  t.N = (long long)nx * ny;
  t.tiles_x = (nx + tx - 1) / tx;
  t.ntiles = t.tiles_x * ((ny + ty - 1) / ty);
  return t;
}

// Per-CTA accumulation of dot products without register arrays: each warp owns one
// row of `wacc`; per tile, a value is warp-reduced and lane 0 adds it to the row.
// Tiles are visited in a fixed order, so the sums are deterministic.
struct WarpAcc {
  double v[NT / 32][NP];
};
__device__ __forceinline__ void wacc_clear(WarpAcc& a) {
  for (int q = threadIdx.x; q < (NT / 32) * NP; q += NT) (&a.v[0][0])[q] = 0.0;
  __syncthreads();
}
__device__ __forceinline__ void wacc_add(WarpAcc& a, int k, double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  if ((threadIdx.x & 31) == 0) a.v[threadIdx.x >> 5][k] += x;
}
// four consecutive slots k..k+3 at once (independent shuffles interleave)
__device__ __forceinline__ void wacc_add4(WarpAcc& a, int k, double (&x)[4]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int u = 0; u < 4; ++u) x[u] += __shfl_xor_sync(0xffffffffu, x[u], o);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int u = 0; u < 4; ++u) a.v[threadIdx.x >> 5][k + u] += x[u];
}
// CTA totals of slots [0, kn) -> out[0, kn)
__device__ __forceinline__ void wacc_store(WarpAcc& a, int kn, double* out) {
  __syncthreads();
  if (threadIdx.x < kn) {
    double sum = 0.0;
    for (int w = 0; w < NT / 32; ++w) sum += a.v[w][threadIdx.x];
    out[threadIdx.x] = sum;
  }
  __syncthreads();
}

// Identical-in-every-CTA reduction of partial[0..nblk)[0..kn) into red[0..kn).
// Slot k is summed unless bit 2k / 2k+1 of `minmax` asks for its minimum / maximum.
// Thread (w, k) combines blocks w, w + 8, w + 16, ... of slot k in increasing order
// (16 loads in flight, consecutive threads read consecutive slots), then the eight
// warp results of each slot are combined in warp order: a fixed order, so every CTA
// and every run gets the same bits.  `tmp` is free CTA scratch of 8 x NP doubles.
enum { RED_SUM = 0, RED_MIN = 1, RED_MAX = 2 };
__device__ __forceinline__ double red_op(int kind, double a, double b) {
  return kind == RED_SUM ? a + b : (kind == RED_MIN ? fmin(a, b) : fmax(a, b));
}
__device__ __forceinline__ double red_init(int kind) {
  return kind == RED_SUM ? 0.0 : (kind == RED_MIN ? INFINITY : -INFINITY);
}
__device__ inline void grid_reduce(const double* partial, int nblk, int kn, double* red, WarpAcc& tmp,
                                   unsigned minmax = 0u) {
  constexpr int NW = NT / 32, U = 16;
  const int k = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int kind = k < 16 ? (int)((minmax >> (2 * k)) & 3u) : RED_SUM;
  double s = red_init(kind);
  if (k < kn) {
    for (int b0 = w; b0 < nblk; b0 += NW * U) {
      double v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int b = b0 + u * NW;
        v[u] = b < nblk ? ldcg(partial + (long long)b * NP + k) : red_init(kind);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) s = red_op(kind, s, v[u]);
    }
  }
  tmp.v[w][k] = s;
  __syncthreads();
  if (threadIdx.x < kn) {
    const int kk = threadIdx.x < 16 ? (int)((minmax >> (2 * threadIdx.x)) & 3u) : RED_SUM;
    double t = red_init(kk);
    for (int q = 0; q < NW; ++q) t = red_op(kk, t, tmp.v[q][threadIdx.x]);
    red[threadIdx.x] = t;
  }
  __syncthreads();
}

// ------------------------------------------------------------------ tiles
// A CTA works on a TX x TY tile of interior cells plus a halo; each thread owns
// CPT cells of the tile (rows ly and ly + RY).  The vector being multiplied and
// the operator's frozen coefficients are staged in shared memory together.
constexpr int RY = NT / TX;     // rows covered by one pass of the CTA
constexpr int CPT = TY / RY;    // interior cells per thread

// The tile shape of an operator: TX x TY, unless the operator names its own (kTileX x
// kTileY, a shape an ensemble's autotuner may choose).  RYo rows per CTA pass, CPTo cells
// per thread.
template <class Op, class = void>
struct TileShape {
  static constexpr int tx = TX, ty = TY;
};
template <class Op>
struct TileShape<Op, std::void_t<decltype(Op::kTileX)>> {
  static constexpr int tx = Op::kTileX, ty = Op::kTileY;
};
template <class Op>
constexpr int TXo = TileShape<Op>::tx;
template <class Op>
constexpr int TYo = TileShape<Op>::ty;
template <class Op>
constexpr int RYo = NT / TXo<Op>;
template <class Op>
constexpr int CPTo = TYo<Op> / RYo<Op>;
template <class Op>
inline Tiling make_tiling_for(const imex_ctx* ctx) {
  return make_tiling(ctx->nx, ctx->ny, ctx->P.xclamp, ctx->P.yclamp, TXo<Op>, TYo<Op>);
}

__device__ __forceinline__ int wrapc(int i, int n) {
  if (i < 0) {
    i += n;
    if (i < 0) i = wrap(i, n);
  } else if (i >= n) {
    i -= n;
    if (i >= n) i = wrap(i, n);
  }
  return i;
}

template <class Op>
struct TileBuf {
  using T = typename Op::value_type;
  static constexpr int H = Op::HALO;
  static constexpr int SX = TXo<Op> + 2 * H, SY = TYo<Op> + 2 * H, SN = SX * SY;
  static constexpr int PX = TXo<Op> + 2, PY = TYo<Op> + 2, PN = PX * PY;  // halo-1 region of the pre-pass
  T s[Op::M * SN];           // vector tile
  T c[Op::QT * SN];          // frozen coefficients on the same cells
  T p[Op::PT * PN + 1];      // pre-pass quantities (halo-1 region)
};

// ------------------------------------------------------------------ operators
// Each operator is a template on its arithmetic type T: double is the plain FP64
// path (the same operations, in the same order, as the reference), float the
// operator of the inner solves of the mixed-precision form.  Coefficients are
// read from the FP64 planes and rounded to T when a tile is staged.
//
// Pressure_Subsystem_AX (implicit_operators.cpp:505-616), GLF or local viscosity,
// with the frozen coefficient planes of one solve; precP (implicit_operators.cpp:650-662).
struct PressureCoef {
  DevParams P;
  const DevScalars* sc;
  const double *hh, *eta, *rho, *vscale, *tdiag, *vdiag;
  const double* lv;  // local dissipation (GLF off): K of the faces x+, x-, y+, y- (k_local_visc), else null
  double h, hh2, idx2, idy2, nu_x, nu_y, cvx, cvy, a;
  int jac;
  // step scalars of the current sub-step (h, GLF viscosity), read from device memory
  __device__ __forceinline__ void bind() {
    h = sc->h;
    hh2 = h * h;
    idx2 = 1 / (P.dx * P.dx);
    idy2 = 1 / (P.dy * P.dy);
    nu_x = 0.0;
    nu_y = 0.0;
    if (P.add_pvisc == IMEX_MaterialSpeedp) {
      nu_x = sc->vx_max * P.dx;
      nu_y = sc->vy_max * P.dy;
    } else if (P.add_pvisc == IMEX_AlfvenSpeedp) {
      nu_x = sc->cA_x * P.dx;
      nu_y = sc->cA_y * P.dy;
    }
    cvx = nu_x / (P.dx * P.dx);  // the reference divides here (implicit_operators.cpp:585)
    cvy = nu_y / (P.dy * P.dy);
    a = 1.0 / (P.gamma - 1.0);
  }
};
template <class T>
struct PressureOpT : PressureCoef {
  using value_type = T;
  static constexpr int M = 1, HALO = 1;
  static constexpr int COEF = 5;  // hh, eta, rho, vscale, tdiag (+ vdiag in J mode)
  static constexpr int QT = 2;    // staged: hh, eta
  static constexpr int PT = 0;
  static constexpr int MIN_BLOCKS = 2;
  // the same operator with arithmetic type U
  template <class U>
  __device__ __forceinline__ PressureOpT<U> as() const {
    PressureOpT<U> o;
    static_cast<PressureCoef&>(o) = *this;
    return o;
  }
  __device__ __forceinline__ void coef(long long c, T* q) const {
    q[0] = (T)__ldg(hh + c);
    q[1] = (T)__ldg(eta + c);
  }
  template <class TB>
  __device__ __forceinline__ void prepass(TB&, int, int) const {}
  template <class TB>
  __device__ __forceinline__ void matvec(const TB& tb, int lx, int ly, long long c, T* out) const {
    const int sx = TB::SX, o = (ly + 1) * sx + lx + 1;
    const T hf = T(0.5);
    const T* x = tb.s;
    const T* hq = tb.c;
    const T* eq = tb.c + TB::SN;
    const T xc = x[o], xe = x[o + 1], xw = x[o - 1], xn = x[o + sx], xs = x[o - sx];
    const T h00 = hq[o], hp0 = hq[o + 1], hm0 = hq[o - 1], h0p = hq[o + sx], h0m = hq[o - sx];
    const T Vd = jac ? (T)__ldcg(vdiag + c) : (T)a;
    T r = Vd * xc - (T)hh2 * ((T)idx2 * (hf * (hp0 + h00) * (xe - xc) - hf * (h00 + hm0) * (xc - xw)) +
                              (T)idy2 * (hf * (h0p + h00) * (xn - xc) - hf * (h0m + h00) * (xc - xs)));
    T lap;
    if (lv) {  // implicit_operators.cpp:584-607
      const long long N = P.N;
      const T kxp = (T)__ldg(lv + c), kxm = (T)__ldg(lv + N + c);
      const T kyp = (T)__ldg(lv + 2 * N + c), kym = (T)__ldg(lv + 3 * N + c);
      lap = (T)idx2 * (kxp * (xe - xc) - kxm * (xc - xw)) + (T)idy2 * (kyp * (xn - xc) - kym * (xc - xs));
    } else {
      const T ec = eq[o], ee = eq[o + 1], ew = eq[o - 1], en = eq[o + sx], es = eq[o - sx];
      lap = (T)cvx * (hf * (ee + ec) * (xe - xc) - hf * (ec + ew) * (xc - xw)) +
            (T)cvy * (hf * (en + ec) * (xn - xc) - hf * (ec + es) * (xc - xs));
    }
    out[0] = r - (T)__ldg(vscale + c) * (T)h * lap;
  }
  __device__ __forceinline__ void precond(long long c, T* v) const {
    const T Vd = jac ? (T)__ldcg(vdiag + c) : (T)a;
    v[0] = v[0] / (Vd + (T)__ldg(tdiag + c));
  }
};
using PressureOp = PressureOpT<double>;

// Energy_Subsystem_AX (implicit_operators.cpp:741-795), periodic, on the total energy E:
//   A E = (E - (g-1) h^2 div(hh grad E)) dx dy,  hh = h(Qe) rho_e / rho frozen per solve;
// precE (imex_subsystems.cpp:487-505) divides by the staged diag dx dy.
struct EnergyCoef {
  DevParams P;
  const DevScalars* sc;
  const double *hh, *tdiag;
  double gh2, idx2, idy2, dx, dy;
  __device__ __forceinline__ void bind() {
    const double h = sc->h;
    gh2 = (P.gamma - 1) * h * h;
    idx2 = 1.0 / (P.dx * P.dx);
    idy2 = 1.0 / (P.dy * P.dy);
    dx = P.dx;
    dy = P.dy;
  }
};
template <class T>
struct EnergyOpT : EnergyCoef {
  using value_type = T;
  static constexpr int M = 1, HALO = 1;
  static constexpr int COEF = 2;  // hh, tdiag
  static constexpr int QT = 1;    // staged: hh
  static constexpr int PT = 0;
  static constexpr int MIN_BLOCKS = 2;
  template <class U>
  __device__ __forceinline__ EnergyOpT<U> as() const {
    EnergyOpT<U> o;
    static_cast<EnergyCoef&>(o) = *this;
    return o;
  }
  __device__ __forceinline__ void coef(long long c, T* q) const { q[0] = (T)__ldg(hh + c); }
  template <class TB>
  __device__ __forceinline__ void prepass(TB&, int, int) const {}
  template <class TB>
  __device__ __forceinline__ void matvec(const TB& tb, int lx, int ly, long long, T* out) const {
    const int sx = TB::SX, o = (ly + 1) * sx + lx + 1;
    const T hf = T(0.5);
    const T* x = tb.s;
    const T* hq = tb.c;
    const T Ei = x[o], xe = x[o + 1], xw = x[o - 1], xn = x[o + sx], xs = x[o - sx];
    const T h00 = hq[o];
    const T hpx = hf * (h00 + hq[o + 1]), hmx = hf * (h00 + hq[o - 1]);
    const T hpy = hf * (h00 + hq[o + sx]), hmy = hf * (h00 + hq[o - sx]);
    const T r = Ei - (T)gh2 * ((T)idx2 * (hpx * (xe - Ei) - hmx * (Ei - xw)) + (T)idy2 * (hpy * (xn - Ei) - hmy * (Ei - xs)));
    out[0] = r * (T)dx * (T)dy;
  }
  __device__ __forceinline__ void precond(long long c, T* v) const { v[0] = v[0] / (T)__ldg(tdiag + c); }
};
using EnergyOp = EnergyOpT<double>;

// Magnetic_Subsystem_AX (implicit_operators.cpp:141-353), GLF or local viscosity.
struct MagneticBCoef {
  DevParams P;
  const DevScalars* sc;
  const double *Qe, *rho;
  const double* lv;  // local dissipation (GLF off): nu of the faces x+, x-, y+, y- (k_local_visc), else null
  double h, nu_x, nu_y, cx, cy;
  __device__ __forceinline__ void bind() {
    h = sc->h;
    nu_x = sc->B_max_x * P.dx;
    nu_y = sc->B_max_y * P.dy;
    cx = nu_x / (P.dx * P.dx);
    cy = nu_y / (P.dy * P.dy);
  }
};
template <class T>
struct MagneticBOpT : MagneticBCoef {
  using value_type = T;
  static constexpr int M = 3, HALO = 1;
  static constexpr int COEF = 4;  // Qe B (3), rho
  static constexpr int QT = 4;    // staged: Qe Bx, By, Bz, rho
  static constexpr int PT = 0;
  static constexpr int MIN_BLOCKS = 1;  // the 9-point stencil keeps many corner averages live
  template <class U>
  __device__ __forceinline__ MagneticBOpT<U> as() const {
    MagneticBOpT<U> o;
    static_cast<MagneticBCoef&>(o) = *this;
    return o;
  }
  __device__ __forceinline__ void coef(long long c, T* q) const {
    q[0] = (T)__ldg(Qe + 5 * P.N + c);
    q[1] = (T)__ldg(Qe + 6 * P.N + c);
    q[2] = (T)__ldg(Qe + 7 * P.N + c);
    q[3] = (T)__ldg(rho + c);
  }
  template <class TB>
  __device__ __forceinline__ void prepass(TB&, int, int) const {}
  __device__ __forceinline__ void precond(long long, T*) const {}
  // the viscous Laplacian of one component x at staged cell o: the GLF form with the global
  // coefficients cxT = B_max_x dx / dx^2, cyT (implicit_operators.cpp:311-320), or the face
  // viscosities of the local form (implicit_operators.cpp:346-352)
  __device__ __forceinline__ T visc(const T* x, long long c, int o, int sx, T cxT, T cyT) const {
    const T two = T(2), one = T(1);
    if (lv) {
      const long long N = P.N;
      const T dx = (T)P.dx, dy = (T)P.dy;
      const T nxp = (T)__ldg(lv + c), nxm = (T)__ldg(lv + N + c);
      const T nyp = (T)__ldg(lv + 2 * N + c), nym = (T)__ldg(lv + 3 * N + c);
      return one / (dx * dx) * (nxp * (x[o + 1] - x[o]) - nxm * (x[o] - x[o - 1])) +
             one / (dy * dy) * (nyp * (x[o + sx] - x[o]) - nym * (x[o] - x[o - sx]));
    }
    return cxT * (x[o - 1] - two * x[o] + x[o + 1]) + cyT * (x[o - sx] - two * x[o] + x[o + sx]);
  }
  template <class TB>
  __device__ void matvec(const TB& tb, int lx, int ly, long long c, T* out) const {
    constexpr int SX = TB::SX, SN = TB::SN;
    const T dx = (T)P.dx, dy = (T)P.dy, hT = (T)h, cxT = (T)cx, cyT = (T)cy;
    const T hf = T(0.5), qf = T(0.25), one = T(1), two = T(2);
    const int o = (ly + 1) * SX + lx + 1;
    // offsets: C, E, W, N, S, NE, SE, NW, SW
    const int E = o + 1, W = o - 1, No = o + SX, S = o - SX, NE = No + 1, SE = S + 1, NW = No - 1, SW = S - 1;
    const T* q5 = tb.c;
    const T* q6 = tb.c + SN;
    const T* q7 = tb.c + 2 * SN;
    const T* rr = tb.c + 3 * SN;
    const T* x5 = tb.s;
    const T* x6 = tb.s + SN;
    const T* x7 = tb.s + 2 * SN;
    const T r0 = rr[o];
    const T rho_p0 = hf * (r0 + rr[E]), rho_m0 = hf * (r0 + rr[W]);
    const T rho_0p = hf * (r0 + rr[No]), rho_0m = hf * (r0 + rr[S]);
    // B/rho on a face: the reference divides in every term; the fast arithmetic takes the
    // four face reciprocals once and multiplies (a few ulp; the exact one keeps the divisions)
    const bool fast = P.fast != 0;
    const T ir_p0 = fast ? one / rho_p0 : T(0), ir_m0 = fast ? one / rho_m0 : T(0);
    const T ir_0p = fast ? one / rho_0p : T(0), ir_0m = fast ? one / rho_0m : T(0);
    auto bor = [&](T b, T rho, T ir) { return fast ? b * ir : b / rho; };
#define FA(a, t) (hf * (a[o] + a[t]))
#define CA(a, t1, t2, t3) (qf * (a[o] + a[t1] + a[t2] + a[t3]))
#define QX(t) (hf * (q5[t] * x5[t] + q6[t] * x6[t] + q7[t] * x7[t]))
    const T Bxn_pp = CA(q5, E, No, NE), Bxn_pm = CA(q5, E, S, SE), Bxn_mp = CA(q5, W, No, NW),
            Bxn_mm = CA(q5, W, S, SW);
    const T Byn_pp = CA(q6, E, No, NE), Byn_pm = CA(q6, E, S, SE), Byn_mp = CA(q6, W, No, NW),
            Byn_mm = CA(q6, W, S, SW);
    const T Bzn_pp = CA(q7, E, No, NE), Bzn_pm = CA(q7, E, S, SE), Bzn_mp = CA(q7, W, No, NW),
            Bzn_mm = CA(q7, W, S, SW);
    const T Bx_pp = CA(x5, E, No, NE), Bx_pm = CA(x5, E, S, SE), Bx_mp = CA(x5, W, No, NW),
            Bx_mm = CA(x5, W, S, SW);
    const T By_pp = CA(x6, E, No, NE), By_pm = CA(x6, E, S, SE), By_mp = CA(x6, W, No, NW),
            By_mm = CA(x6, W, S, SW);
    const T Bz_pp = CA(x7, E, No, NE), Bz_pm = CA(x7, E, S, SE), Bz_mp = CA(x7, W, No, NW),
            Bz_mm = CA(x7, W, S, SW);
    // the energy-like corner sums shared by several terms
    const T Wpp = hf * (Bxn_pp * Bx_pp + Byn_pp * By_pp + Bzn_pp * Bz_pp);
    const T Wpm = hf * (Bxn_pm * Bx_pm + Byn_pm * By_pm + Bzn_pm * Bz_pm);
    const T Wmp = hf * (Bxn_mp * Bx_mp + Byn_mp * By_mp + Bzn_mp * Bz_mp);
    const T Wmm = hf * (Bxn_mm * Bx_mm + Byn_mm * By_mm + Bzn_mm * Bz_mm);
    const T QXc = QX(o);
    {  // x component (implicit_operators.cpp:266-275)
      const T QXn = QX(No), QXs = QX(S);
      const T Bx_1 = bor(FA(q5, No), rho_0p, ir_0p) *
                     (one / dx * (Bxn_pp * By_pp - Bxn_mp * By_mp) -
                      one / dy * ((QXn - q6[No] * x6[No]) - (QXc - q6[o] * x6[o])));
      const T Bx_2 = bor(FA(q6, No), rho_0p, ir_0p) *
                     (one / dx * ((Wpp - Bxn_pp * Bx_pp) - (Wmp - Bxn_mp * Bx_mp)) -
                      one / dy * (q6[No] * x5[No] - q6[o] * x5[o]));
      const T Bx_3 = bor(FA(q5, S), rho_0m, ir_0m) *
                     (one / dx * (Bxn_pm * By_pm - Bxn_mm * By_mm) -
                      one / dy * ((QXc - q6[o] * x6[o]) - (QXs - q6[S] * x6[S])));
      const T Bx_4 = bor(FA(q6, S), rho_0m, ir_0m) *
                     (one / dx * ((Wpm - Bxn_pm * Bx_pm) - (Wmm - Bxn_mm * Bx_mm)) -
                      one / dy * (q6[o] * x5[o] - q6[S] * x5[S]));
      const T ax5 = x5[o] + (hT * hT / dy) * ((Bx_1 + Bx_2) - (Bx_3 + Bx_4));
      out[0] = ax5 - hT * visc(x5, c, o, SX, cxT, cyT);
    }
    const T QXe = QX(E), QXw = QX(W);
    {  // y component (implicit_operators.cpp:277-285)
      const T By_1 = bor(FA(q6, E), rho_p0, ir_p0) *
                     (-one / dx * ((QXe - q5[E] * x5[E]) - (QXc - q5[o] * x5[o])) +
                      one / dy * (Bxn_pp * By_pp - Bxn_pm * By_pm));
      const T By_2 = bor(FA(q5, E), rho_p0, ir_p0) *
                     (-one / dx * (q5[E] * x6[E] - q5[o] * x6[o]) +
                      one / dy * ((Wpp - Byn_pp * By_pp) - (Wpm - Byn_pm * By_pm)));
      const T By_3 = bor(FA(q6, W), rho_m0, ir_m0) *
                     (-one / dx * ((QXc - q5[o] * x5[o]) - (QXw - q5[W] * x5[W])) +
                      one / dy * (Bxn_mp * By_mp - Bxn_mm * By_mm));
      const T By_4 = bor(FA(q5, W), rho_m0, ir_m0) *
                     (-one / dx * (q5[o] * x6[o] - q5[W] * x6[W]) +
                      one / dy * ((Wmp - Byn_mp * By_mp) - (Wmm - Byn_mm * By_mm)));
      const T ax6 = x6[o] + (hT * hT / dx) * ((By_1 + By_2) - (By_3 + By_4));
      out[1] = ax6 - hT * visc(x6, c, o, SX, cxT, cyT);
    }
    {  // z component (implicit_operators.cpp:288-306)
      const T QXn = QX(No), QXs = QX(S);
      const T Bz_1 = bor(FA(q7, E), rho_p0, ir_p0) *
                     (-one / dx * ((QXe - q5[E] * x5[E]) - (QXc - q5[o] * x5[o])) +
                      one / dy * (Byn_pp * Bx_pp - Byn_pm * Bx_pm));
      const T Bz_2 = bor(FA(q5, E), rho_p0, ir_p0) *
                     (-one / dx * (q5[E] * x7[E] - q5[o] * x7[o]) - one / dy * (Byn_pp * Bz_pp - Byn_pm * Bz_pm));
      const T Bz_3 = bor(FA(q7, W), rho_m0, ir_m0) *
                     (-one / dx * ((QXc - q5[o] * x5[o]) - (QXw - q5[W] * x5[W])) +
                      one / dy * (Byn_mp * Bx_mp - Byn_mm * Bx_mm));
      const T Bz_4 = bor(FA(q5, W), rho_m0, ir_m0) *
                     (-one / dx * (q5[o] * x7[o] - q5[W] * x7[W]) - one / dy * (Byn_mp * Bz_mp - Byn_mm * Bz_mm));
      const T Bz_5 = bor(FA(q7, No), rho_0p, ir_0p) *
                     (one / dx * (Bxn_pp * By_pp - Bxn_mp * By_mp) -
                      one / dy * ((QXn - q6[No] * x6[No]) - (QXc - q6[o] * x6[o])));
      const T Bz_6 = bor(FA(q6, No), rho_0p, ir_0p) *
                     (-one / dx * (Bxn_pp * Bz_pp - Bxn_mp * Bz_mp) - one / dy * (q6[No] * x7[No] - q6[o] * x7[o]));
      const T Bz_7 = bor(FA(q7, S), rho_0m, ir_0m) *
                     (one / dx * (Bxn_pm * By_pm - Bxn_mm * By_mm) -
                      one / dy * ((QXc - q6[o] * x6[o]) - (QXs - q6[S] * x6[S])));
      const T Bz_8 = bor(FA(q6, S), rho_0m, ir_0m) *
                     (-one / dx * (Bxn_pm * Bz_pm - Bxn_mm * Bz_mm) - one / dy * (q6[o] * x7[o] - q6[S] * x7[S]));
      const T ax7 =
          x7[o] + hT * hT / dx * ((Bz_1 + Bz_2) - (Bz_3 + Bz_4)) + hT * hT / dy * ((Bz_5 + Bz_6) - (Bz_7 + Bz_8));
      out[2] = ax7 - hT * visc(x7, c, o, SX, cxT, cyT);
    }
#undef FA
#undef CA
#undef QX
  }
};
using MagneticBOp = MagneticBOpT<double>;

// Magnetic_Subsystem_AX in the fast arithmetic (imex_config.arith = fast).  The exact form
// above evaluates each corner average of Qe B and of x from the cell's own side, four
// corners per cell, so every corner is formed four times and its 28 corner quantities stay
// live through the three components (226-240 registers: one CTA per SM).  Here a tile
// pre-pass forms, once per corner, the corner averages of Qe B and of x (in the reference's
// order for the corner's lower-left cell, whose upper-right corner it is) and their
// energy-like sum W, and once per staged cell the sum QX = (q5 x5 + q6 x6 + q7 x7) / 2; the
// matvec reads them from shared memory.  The corners seen from the other three cells round
// their four-term sums in another order, a few ulp from the reference's operator; the
// solves converge to the same tolerance.  It fits two CTAs per SM.
template <class T, int kTX = TX, int kTY = TY>
struct MagneticBFastOpT : MagneticBOpT<T> {
  static constexpr int kTileX = kTX, kTileY = kTY;
  using MagneticBCoef::P;
  using MagneticBCoef::h;
  using MagneticBCoef::cx;
  using MagneticBCoef::cy;
  // pre-pass planes: corners (indexed by their lower-left staged cell) Bxn, Byn, Bzn, Bx, By,
  // Bz, W; and QX at every staged cell
  static constexpr int PT = 8;
  static constexpr int MIN_BLOCKS = 2;
  template <class U>
  __device__ __forceinline__ MagneticBFastOpT<U, kTX, kTY> as() const {
    MagneticBFastOpT<U, kTX, kTY> o;
    static_cast<MagneticBCoef&>(o) = *this;
    return o;
  }
  template <class TB>
  __device__ __forceinline__ void prepass(TB& tb, int, int) const {
    constexpr int SX = TB::SX, SY = TB::SY, SN = TB::SN, PN = TB::PN;
    static_assert(TB::PN == TB::SN, "halo-1 tile: the pre-pass region is the staged region");
    const T hf = T(0.5), qf = T(0.25);
    const T* q5 = tb.c;
    const T* q6 = tb.c + SN;
    const T* q7 = tb.c + 2 * SN;
    const T* x5 = tb.s;
    const T* x6 = tb.s + SN;
    const T* x7 = tb.s + 2 * SN;
    for (int q = threadIdx.x; q < SN; q += NT) {
      tb.p[7 * PN + q] = hf * (q5[q] * x5[q] + q6[q] * x6[q] + q7[q] * x7[q]);
      const int sx = q % SX, sy = q / SX;
      if (sx >= SX - 1 || sy >= SY - 1) continue;  // no upper-right neighbours: not a corner
      const int e = q + 1, n = q + SX, ne = q + SX + 1;
      const T bxn = qf * (q5[q] + q5[e] + q5[n] + q5[ne]);
      const T byn = qf * (q6[q] + q6[e] + q6[n] + q6[ne]);
      const T bzn = qf * (q7[q] + q7[e] + q7[n] + q7[ne]);
      const T bx = qf * (x5[q] + x5[e] + x5[n] + x5[ne]);
      const T by = qf * (x6[q] + x6[e] + x6[n] + x6[ne]);
      const T bz = qf * (x7[q] + x7[e] + x7[n] + x7[ne]);
      tb.p[0 * PN + q] = bxn;
      tb.p[1 * PN + q] = byn;
      tb.p[2 * PN + q] = bzn;
      tb.p[3 * PN + q] = bx;
      tb.p[4 * PN + q] = by;
      tb.p[5 * PN + q] = bz;
      tb.p[6 * PN + q] = hf * (bxn * bx + byn * by + bzn * bz);
    }
  }
  // implicit_operators.cpp:214-353 with the corner quantities of the pre-pass: the corners
  // (i +- 1/2, j +- 1/2) of cell o are the pre-pass entries of o (pp), S (pm), W (mp), SW (mm)
  template <class TB>
  __device__ void matvec(const TB& tb, int lx, int ly, long long c, T* out) const {
    constexpr int SX = TB::SX, SN = TB::SN, PN = TB::PN;
    const T dx = (T)P.dx, dy = (T)P.dy, hT = (T)h, cxT = (T)cx, cyT = (T)cy;
    const T hf = T(0.5), one = T(1);
    const int o = (ly + 1) * SX + lx + 1;
    const int E = o + 1, W = o - 1, No = o + SX, S = o - SX, SW = S - 1;
    const T* q5 = tb.c;
    const T* q6 = tb.c + SN;
    const T* q7 = tb.c + 2 * SN;
    const T* rr = tb.c + 3 * SN;
    const T* x5 = tb.s;
    const T* x6 = tb.s + SN;
    const T* x7 = tb.s + 2 * SN;
    const T* Cxn = tb.p;
    const T* Cyn = tb.p + PN;
    const T* Czn = tb.p + 2 * PN;
    const T* Cx = tb.p + 3 * PN;
    const T* Cy = tb.p + 4 * PN;
    const T* Cz = tb.p + 5 * PN;
    const T* Cw = tb.p + 6 * PN;
    const T* QX = tb.p + 7 * PN;
    const T r0 = rr[o];
    const T ir_p0 = one / (hf * (r0 + rr[E])), ir_m0 = one / (hf * (r0 + rr[W]));
    const T ir_0p = one / (hf * (r0 + rr[No])), ir_0m = one / (hf * (r0 + rr[S]));
    const T idx = one / dx, idy = one / dy;
#define FA(a, t) (hf * (a[o] + a[t]))
    {  // x component (implicit_operators.cpp:266-275)
      const T Bx_1 = FA(q5, No) * ir_0p *
                     (idx * (Cxn[o] * Cy[o] - Cxn[W] * Cy[W]) -
                      idy * ((QX[No] - q6[No] * x6[No]) - (QX[o] - q6[o] * x6[o])));
      const T Bx_2 = FA(q6, No) * ir_0p *
                     (idx * ((Cw[o] - Cxn[o] * Cx[o]) - (Cw[W] - Cxn[W] * Cx[W])) -
                      idy * (q6[No] * x5[No] - q6[o] * x5[o]));
      const T Bx_3 = FA(q5, S) * ir_0m *
                     (idx * (Cxn[S] * Cy[S] - Cxn[SW] * Cy[SW]) -
                      idy * ((QX[o] - q6[o] * x6[o]) - (QX[S] - q6[S] * x6[S])));
      const T Bx_4 = FA(q6, S) * ir_0m *
                     (idx * ((Cw[S] - Cxn[S] * Cx[S]) - (Cw[SW] - Cxn[SW] * Cx[SW])) -
                      idy * (q6[o] * x5[o] - q6[S] * x5[S]));
      const T ax5 = x5[o] + (hT * hT / dy) * ((Bx_1 + Bx_2) - (Bx_3 + Bx_4));
      out[0] = ax5 - hT * this->visc(x5, c, o, SX, cxT, cyT);
    }
    {  // y component (implicit_operators.cpp:277-285)
      const T By_1 = FA(q6, E) * ir_p0 *
                     (-idx * ((QX[E] - q5[E] * x5[E]) - (QX[o] - q5[o] * x5[o])) +
                      idy * (Cxn[o] * Cy[o] - Cxn[S] * Cy[S]));
      const T By_2 = FA(q5, E) * ir_p0 *
                     (-idx * (q5[E] * x6[E] - q5[o] * x6[o]) +
                      idy * ((Cw[o] - Cyn[o] * Cy[o]) - (Cw[S] - Cyn[S] * Cy[S])));
      const T By_3 = FA(q6, W) * ir_m0 *
                     (-idx * ((QX[o] - q5[o] * x5[o]) - (QX[W] - q5[W] * x5[W])) +
                      idy * (Cxn[W] * Cy[W] - Cxn[SW] * Cy[SW]));
      const T By_4 = FA(q5, W) * ir_m0 *
                     (-idx * (q5[o] * x6[o] - q5[W] * x6[W]) +
                      idy * ((Cw[W] - Cyn[W] * Cy[W]) - (Cw[SW] - Cyn[SW] * Cy[SW])));
      const T ax6 = x6[o] + (hT * hT / dx) * ((By_1 + By_2) - (By_3 + By_4));
      out[1] = ax6 - hT * this->visc(x6, c, o, SX, cxT, cyT);
    }
    {  // z component (implicit_operators.cpp:288-306)
      const T Bz_1 = FA(q7, E) * ir_p0 *
                     (-idx * ((QX[E] - q5[E] * x5[E]) - (QX[o] - q5[o] * x5[o])) +
                      idy * (Cyn[o] * Cx[o] - Cyn[S] * Cx[S]));
      const T Bz_2 = FA(q5, E) * ir_p0 *
                     (-idx * (q5[E] * x7[E] - q5[o] * x7[o]) - idy * (Cyn[o] * Cz[o] - Cyn[S] * Cz[S]));
      const T Bz_3 = FA(q7, W) * ir_m0 *
                     (-idx * ((QX[o] - q5[o] * x5[o]) - (QX[W] - q5[W] * x5[W])) +
                      idy * (Cyn[W] * Cx[W] - Cyn[SW] * Cx[SW]));
      const T Bz_4 = FA(q5, W) * ir_m0 *
                     (-idx * (q5[o] * x7[o] - q5[W] * x7[W]) - idy * (Cyn[W] * Cz[W] - Cyn[SW] * Cz[SW]));
      const T Bz_5 = FA(q7, No) * ir_0p *
                     (idx * (Cxn[o] * Cy[o] - Cxn[W] * Cy[W]) -
                      idy * ((QX[No] - q6[No] * x6[No]) - (QX[o] - q6[o] * x6[o])));
      const T Bz_6 = FA(q6, No) * ir_0p *
                     (-idx * (Cxn[o] * Cz[o] - Cxn[W] * Cz[W]) - idy * (q6[No] * x7[No] - q6[o] * x7[o]));
      const T Bz_7 = FA(q7, S) * ir_0m *
                     (idx * (Cxn[S] * Cy[S] - Cxn[SW] * Cy[SW]) -
                      idy * ((QX[o] - q6[o] * x6[o]) - (QX[S] - q6[S] * x6[S])));
      const T Bz_8 = FA(q6, S) * ir_0m *
                     (-idx * (Cxn[S] * Cz[S] - Cxn[SW] * Cz[SW]) - idy * (q6[o] * x7[o] - q6[S] * x7[S]));
      const T ax7 =
          x7[o] + hT * hT / dx * ((Bz_1 + Bz_2) - (Bz_3 + Bz_4)) + hT * hT / dy * ((Bz_5 + Bz_6) - (Bz_7 + Bz_8));
      out[2] = ax7 - hT * this->visc(x7, c, o, SX, cxT, cyT);
    }
#undef FA
  }
};
using MagneticBFastOp = MagneticBFastOpT<double>;

// Magnetic_Subsystem_potential_AX (implicit_operators.cpp:355-503), GLF or local viscosity.
// The reference evaluates B = curl A and the stress tensor T^B at the four
// neighbours of each cell; those values are exactly curl A and T^B of the
// neighbouring cells, so the tile pre-pass computes them once per cell (same
// arithmetic) and the per-cell pass only differences them.
struct MagneticACoef {
  DevParams P;
  const DevScalars* sc;
  const double *Qe, *rho;
  const double* irho;  // fast arithmetic: 1/rho (from k_magnetic_rhs_A, or k_recip for a prepared operator), else null
  const double* lv;  // local dissipation (GLF off): nu of the faces x+, x-, y+, y- (k_local_visc), else null
  double h, nu_x, nu_y, cx, cy;
  int add_bvisc;
  __device__ __forceinline__ void bind() {
    h = sc->h;
    nu_x = sc->gmax_bx * P.dx;
    nu_y = sc->gmax_by * P.dy;
    cx = nu_x / (P.dx * P.dx);
    cy = nu_y / (P.dy * P.dy);
  }
};
// kOpen: an instance for runs with a transmissive direction, whose tiles extrapolate A
// past the domain (extrapolate); the periodic instance carries none of that code.
template <class T, bool kOpen = false>
struct MagneticAOpT : MagneticACoef {
  using value_type = T;
  static constexpr int M = 3, HALO = 2;
  static constexpr int COEF = 4;  // Qe B (3), rho
  static constexpr int QT = 3;    // staged: Qe Bx, By, Bz
  static constexpr int PT = 6;    // Txx, Tyx, Tzx, Txy, Tyy, Tzy on the halo-1 region
  static constexpr int MIN_BLOCKS = 2;
  template <class U>
  __device__ __forceinline__ MagneticAOpT<U, kOpen> as() const {
    MagneticAOpT<U, kOpen> o;
    static_cast<MagneticACoef&>(o) = *this;
    return o;
  }
  __device__ __forceinline__ void coef(long long c, T* q) const {
    q[0] = (T)__ldg(Qe + 5 * P.N + c);
    q[1] = (T)__ldg(Qe + 6 * P.N + c);
    q[2] = (T)__ldg(Qe + 7 * P.N + c);
  }
  __device__ __forceinline__ void precond(long long, T*) const {}
  // bound_cond_A on the staged vector: the operator reads AG = bound_cond_A(x)
  // (implicit_operators.cpp:377-384).  In a transmissive direction the staged cells outside
  // the domain get linear extrapolations of the two nearest interior cells (boundary.cpp:
  // 181-195, 233-246), x first, then y on the x-extrapolated rows; the fill left the
  // clamped values there.  Tiles away from such a boundary have nothing to do.
  template <class TB>
  __device__ __forceinline__ void extrapolate(TB& tb, int x0, int y0) const {
    constexpr int SX = TB::SX, SY = TB::SY, SN = TB::SN, H = HALO;
    if (P.xclamp && (x0 - H < 0 || x0 - H + SX > P.nx)) {
      const int sa = H - x0, sr = P.nx - 1 - x0 + H;  // staged columns of i = 0 and i = nx - 1
      for (int q = threadIdx.x; q < SN; q += NT) {
        const int sx = q % SX, gi = x0 - H + sx;
        if (gi >= 0 && gi < P.nx) continue;
        T* r = tb.s + (q - sx);
#pragma unroll
        for (int m = 0; m < M; ++m, r += SN) {
          if (gi < 0) {
            const T slope = r[sa + 1] - r[sa];
            r[sx] = r[sa] - (T)(-gi) * slope;
          } else {
            const T slope = r[sr] - r[sr - 1];
            r[sx] = r[sr] + (T)(gi - P.nx + 1) * slope;
          }
        }
      }
      __syncthreads();
    }
    if (P.yclamp && (y0 - H < 0 || y0 - H + SY > P.ny)) {
      const int ra = H - y0, rt = P.ny - 1 - y0 + H;  // staged rows of j = 0 and j = ny - 1
      for (int q = threadIdx.x; q < SN; q += NT) {
        const int sx = q % SX, sy = q / SX, gj = y0 - H + sy;
        if (gj >= 0 && gj < P.ny) continue;
        T* c = tb.s + sx;
#pragma unroll
        for (int m = 0; m < M; ++m, c += SN) {
          if (gj < 0) {
            const T slope = c[(ra + 1) * SX] - c[ra * SX];
            c[sy * SX] = c[ra * SX] - (T)(-gj) * slope;
          } else {
            const T slope = c[rt * SX] - c[(rt - 1) * SX];
            c[sy * SX] = c[rt * SX] + (T)(gj - P.ny + 1) * slope;
          }
        }
      }
      __syncthreads();
    }
  }
  template <class TB>
  __device__ __forceinline__ void prepass(TB& tb, int x0, int y0) const {
    constexpr int SX = TB::SX, SN = TB::SN;
    const T dx = (T)P.dx, dy = (T)P.dy, two = T(2);
    // central differences: a division by 2 dx in the reference; the fast arithmetic multiplies
    // by the reciprocal taken once
    const bool fast = P.fast != 0;
    const T r2dx = T(1) / (two * dx), r2dy = T(1) / (two * dy);
    auto cdx = [&](T d) { return fast ? d * r2dx : d / (two * dx); };
    auto cdy = [&](T d) { return fast ? d * r2dy : d / (two * dy); };
    if constexpr (kOpen) extrapolate(tb, x0, y0);
    for (int q = threadIdx.x; q < TB::PN; q += NT) {
      const int px = q % TB::PX, py = q / TB::PX;
      const int o = (py + 1) * SX + (px + 1);  // same cell in the halo-2 tile
      const T* A0 = tb.s;
      const T* A1 = tb.s + SN;
      const T* A2 = tb.s + 2 * SN;
      const T bx = cdy(A2[o + SX] - A2[o - SX]);
      const T by = cdx(-(A2[o + 1] - A2[o - 1]));
      const T bz = cdx(A1[o + 1] - A1[o - 1]) - cdy(A0[o + SX] - A0[o - SX]);
      const T Bx = tb.c[o], By = tb.c[SN + o], Bz = tb.c[2 * SN + o];
      const T bdot = Bx * bx + By * by + Bz * bz;
      tb.p[0 * TB::PN + q] = bdot / two - Bx * bx;  // Txx
      tb.p[1 * TB::PN + q] = -Bx * by;              // Tyx
      tb.p[2 * TB::PN + q] = -Bx * bz;              // Tzx
      tb.p[3 * TB::PN + q] = -By * bx;              // Txy
      tb.p[4 * TB::PN + q] = bdot / two - By * by;  // Tyy
      tb.p[5 * TB::PN + q] = -By * bz;              // Tzy
    }
  }
  template <class TB>
  __device__ void matvec(const TB& tb, int lx, int ly, long long c, T* out) const {
    constexpr int SX = TB::SX, SN = TB::SN, PX = TB::PX, PN = TB::PN;
    const T dx = (T)P.dx, dy = (T)P.dy, hT = (T)h, two = T(2);
    const int o = (ly + 2) * SX + lx + 2;  // halo-2 tile
    const int p = (ly + 1) * PX + lx + 1;  // halo-1 pre-pass region
    const T* Tq = tb.p;
    const bool fast = P.fast != 0;
    const T r2dx = T(1) / (two * dx), r2dy = T(1) / (two * dy);
    auto cdx = [&](T d) { return fast ? d * r2dx : d / (two * dx); };
    auto cdy = [&](T d) { return fast ? d * r2dy : d / (two * dy); };
    const T divT_x = cdx(Tq[0 * PN + p + 1] - Tq[0 * PN + p - 1]) + cdy(Tq[3 * PN + p + PX] - Tq[3 * PN + p - PX]);
    const T divT_y = cdx(Tq[1 * PN + p + 1] - Tq[1 * PN + p - 1]) + cdy(Tq[4 * PN + p + PX] - Tq[4 * PN + p - PX]);
    const T divT_z = cdx(Tq[2 * PN + p + 1] - Tq[2 * PN + p - 1]) + cdy(Tq[5 * PN + p + PX] - Tq[5 * PN + p - PX]);
    const T hr = irho ? hT * (T)__ldg(irho + c) : hT / (T)__ldg(rho + c);
    const T Fx = hr * divT_x, Fy = hr * divT_y, Fz = hr * divT_z;
    const T Bx = tb.c[o], By = tb.c[SN + o], Bz = tb.c[2 * SN + o];
    const T cross_x = By * Fz - Bz * Fy;
    const T cross_y = Bz * Fx - Bx * Fz;
    const T cross_z = Bx * Fy - By * Fx;
    T nxp = T(0), nxm = T(0), nyp = T(0), nym = T(0);
    if (lv && add_bvisc) {
      const long long N = P.N;
      nxp = (T)__ldg(lv + c);
      nxm = (T)__ldg(lv + N + c);
      nyp = (T)__ldg(lv + 2 * N + c);
      nym = (T)__ldg(lv + 3 * N + c);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T* A = tb.s + k * SN;
      T lap = T(0);
      if (add_bvisc && lv)  // implicit_operators.cpp:481-490
        lap = T(1) / (dx * dx) * (nxp * (A[o + 1] - A[o]) - nxm * (A[o] - A[o - 1])) +
              T(1) / (dy * dy) * (nyp * (A[o + SX] - A[o]) - nym * (A[o] - A[o - SX]));
      else if (add_bvisc)
        lap = (T)cx * (A[o - 1] - two * A[o] + A[o + 1]) + (T)cy * (A[o - SX] - two * A[o] + A[o + SX]);
      const T cr = k == 0 ? cross_x : (k == 1 ? cross_y : cross_z);
      out[k] = A[o] - hT * cr - hT * lap;
    }
  }
};
using MagneticAOp = MagneticAOpT<double>;
using MagneticAOpOpen = MagneticAOpT<double, true>;

template <class Op>
__device__ __forceinline__ bool op_uses_vdiag(const Op&) { return false; }
template <class T>
__device__ __forceinline__ bool op_uses_vdiag(const PressureOpT<T>& o) { return o.jac != 0; }

// ------------------------------------------------------------------ GMRES
template <class TS>
struct GmresWorkT {
  TS *V, *AV;  // Krylov basis (kmax + 1 vectors) and the A v ring (2 vectors)
  double* partial;
  SyncState* sync;
  DevStats* st;
  int kmax, max_restarts;
  int nblk, first;  // the solve's CTAs: [first, first + nblk) of the launch (the whole grid unless batched)
  int fam;  // profile family whose algorithmic bytes this solve accumulates
  double tol, tol_abs;  // stop when |r| <= tol * |r0| + tol_abs
  Tiling T;
};
using GmresWork = GmresWorkT<double>;

// rank of this CTA within the CTAs of its solve
template <class W>
__device__ __forceinline__ int grank(const W& g) {
  return (int)blockIdx.x - g.first;
}

struct GmresShared {
  double H[KCAP + 2][KCAP + 2];
  double cs[KCAP + 2], sn[KCAP + 2], gam[KCAP + 2], alpha[KCAP + 2], sigma[KCAP + 2];
  double red[NP];
  WarpAcc acc;
  int nalpha;  // terms of an update left to the caller (deferred mode), else 0
};

// Stage the vector and the operator's coefficients on the tile at (x0, y0) plus
// halo, then run the operator's pre-pass.  Each thread stages FillQ<Op> cells and
// issues all of their loads before using any: f(c, v) receives the thread's cell
// indices c[FillQ] and fills v[FillQ][M] for all of them at once.
template <class Op>
constexpr int FillQ = (TileBuf<Op>::SN + NT - 1) / NT;

template <class Op, class F>
__device__ __forceinline__ void fill_tile(const Op& op, TileBuf<Op>& tb, const Tiling& T, int x0, int y0, F f) {
  using TB = TileBuf<Op>;
  using VT = typename Op::value_type;
  constexpr int Q = FillQ<Op>;
  constexpr int QC = Op::QT > 0 ? Op::QT : 1;
  long long c[Q];
#pragma unroll
  for (int r = 0; r < Q; ++r) {
    int q = threadIdx.x + r * NT;
    if (q >= TB::SN) q = TB::SN - 1;  // an already staged cell: loaded again, never stored
    const int sxq = q % TB::SX, syq = q / TB::SX;
    int gi = x0 + sxq - Op::HALO, gj = y0 + syq - Op::HALO;
    if (gi < 0 || gi >= T.nx) gi = T.xclamp ? (gi < 0 ? 0 : T.nx - 1) : wrapc(gi, T.nx);
    if (gj < 0 || gj >= T.ny) gj = T.yclamp ? (gj < 0 ? 0 : T.ny - 1) : wrapc(gj, T.ny);
    c[r] = (long long)gi + (long long)T.nx * gj;
  }
  VT qv[Q][QC];
#pragma unroll
  for (int r = 0; r < Q; ++r) op.coef(c[r], qv[r]);
  VT v[Q][Op::M];
  f(c, v);
#pragma unroll
  for (int r = 0; r < Q; ++r) {
    const int q = threadIdx.x + r * NT;
    if (q < TB::SN) {
#pragma unroll
      for (int m = 0; m < Op::M; ++m) tb.s[m * TB::SN + q] = v[r][m];
#pragma unroll
      for (int m = 0; m < Op::QT; ++m) tb.c[m * TB::SN + q] = qv[r][m];
    }
  }
  __syncthreads();
  if (Op::PT > 0) {
    op.prepass(tb, x0, y0);
    __syncthreads();
  }
}

// interior cell r of this thread in the tile at (x0, y0)
struct Cell {
  int lx, ly, gi, gj;
  long long c;
  bool in;
};
template <class Op>
__device__ __forceinline__ Cell tile_cell(const Tiling& T, int x0, int y0, int r) {
  Cell k;
  k.lx = threadIdx.x % TXo<Op>;
  k.ly = threadIdx.x / TXo<Op> + r * RYo<Op>;
  k.gi = x0 + k.lx;
  k.gj = y0 + k.ly;
  k.in = k.gi < T.nx && k.gj < T.ny;
  k.c = (long long)k.gi + (long long)T.nx * k.gj;
  return k;
}

// Result codes of gmres_device
enum { GM_CONVERGED = 0, GM_MAXIT = 1, GM_NONFINITE = 2, GM_SYNC = 3 };

// x_zero: x is treated as zero on entry (its contents are never read), so the first
//   cycle's residual is M^-1 b, a per-cell quantity: it is formed while staging the
//   first matvec tile, and the residual pass and the A v_0 pass become one pass.
// defer: when the solve converges, the last cycle's update sum_i alpha_i v_i is not
//   written; S.alpha[0..S.nalpha) and S.sigma stay in shared memory for the caller to
//   apply in its next pass (the basis stays in g.V).  x_written reports whether an
//   earlier cycle wrote x, in which case the full update is x + that sum.
template <class Op, class TS>
__device__ int gmres_device(const Op& op, const GmresWorkT<TS>& g, double* x, const double* b, GmresShared& S,
                            TileBuf<Op>& tb, unsigned& phase, bool x_zero, bool defer, bool& x_written) {
  using TB = TileBuf<Op>;
  using VT = typename Op::value_type;  // arithmetic of the operator and the staged tile
  constexpr int M = Op::M, HALO = Op::HALO, FQ = FillQ<Op>;
  const Tiling& T = g.T;
  const long long N = T.N;
  const int kmax = g.kmax;
  double tol_eff = g.tol;
  int iters = 0;
  auto Vp = [&](int i) { return g.V + (long long)i * M * N; };
  auto AVp = [&](int i) { return g.AV + (long long)(i & 1) * M * N; };
  auto part = [&]() { return g.partial + (long long)(phase & 1) * g.nblk * NP; };
  const bool lead = threadIdx.x == 0 && grank(g) == 0;
  const int coef = Op::COEF + (op_uses_vdiag(op) ? 1 : 0);
  // algorithmic bytes of a pass that moves `vals` vector values (of type TS) and `cvals`
  // doubles per cell
  auto count = [&](int vals, int cvals) {
    if (lead) g.st->alg_bytes[g.fam] += ((double)vals * sizeof(TS) + (double)cvals * 8.0) * (double)N;
  };
  (void)HALO;
  x_written = false;
  if (threadIdx.x == 0) S.nalpha = 0;

  for (int outer = 0; outer < g.max_restarts; ++outer) {
    const bool from_zero = x_zero && outer == 0;
    const bool last_cycle = outer + 1 >= g.max_restarts;
    if (from_zero) {
      // ---- r0 = M^-1 b -> V0 and Av0 = M^-1 A V0 in one pass; |r0|^2 and r0.Av0
      wacc_clear(S.acc);
      for (int t = grank(g); t < T.ntiles; t += g.nblk) {
        const int x0 = (t % T.tiles_x) * TXo<Op>, y0 = (t / T.tiles_x) * TYo<Op>;
        fill_tile(op, tb, T, x0, y0, [&](const long long* c, VT (*v)[M]) {
#pragma unroll
          for (int r = 0; r < FQ; ++r)
#pragma unroll
            for (int m = 0; m < M; ++m) v[r][m] = (VT)ldcg(b + m * N + c[r]);
#pragma unroll
          for (int r = 0; r < FQ; ++r) op.precond(c[r], v[r]);
        });
        double rr = 0.0, va = 0.0;
#pragma unroll
        for (int r = 0; r < CPTo<Op>; ++r) {
          const Cell k = tile_cell<Op>(T, x0, y0, r);
          if (!k.in) continue;
          VT aw[M];
          op.matvec(tb, k.lx, k.ly, k.c, aw);
          op.precond(k.c, aw);
          const int o = (k.ly + Op::HALO) * TB::SX + k.lx + Op::HALO;
#pragma unroll
          for (int m = 0; m < M; ++m) {
            const double w = (double)tb.s[m * TB::SN + o];
            Vp(0)[m * N + k.c] = (TS)w;
            AVp(0)[m * N + k.c] = (TS)aw[m];
            rr += w * w;
            va += w * (double)aw[m];
          }
        }
        wacc_add(S.acc, 0, rr);
        wacc_add(S.acc, 1, va);
        __syncthreads();
      }
      wacc_store(S.acc, 2, part() + (long long)grank(g) * NP);
      if (!grid_barrier(g.sync, g.nblk)) return GM_SYNC;
      grid_reduce(part(), g.nblk, 2, S.red, S.acc);
      ++phase;
      count(2 * M, M + coef);
      S.gam[0] = sqrt(S.red[0]);
      tol_eff = g.tol * S.gam[0] + g.tol_abs;
      if (!isfinite(S.gam[0])) return GM_NONFINITE;
      if (S.gam[0] <= tol_eff) {
        if (lead) {
          g.st->gmres_iters += iters;
          g.st->last_residual = S.gam[0];
        }
        if (!defer) {  // x = 0
          for (long long c = grank(g) * (long long)NT + threadIdx.x; c < (long long)M * N; c += (long long)g.nblk * NT)
            x[c] = 0.0;
          x_written = true;
        }
        return GM_CONVERGED;
      }
      if (lead) g.st->gmres_restarts += 1;
      S.sigma[0] = 1.0 / S.gam[0];
      for (int r = threadIdx.x; r < (KCAP + 2) * (KCAP + 2); r += NT) (&S.H[0][0])[r] = 0.0;
      __syncthreads();
      if (threadIdx.x == 0) S.H[0][0] = S.sigma[0] * S.sigma[0] * S.red[1];
      __syncthreads();
    } else {
      // ---- residual r0 = M^-1 (b - A x) -> V0, |r0|^2
      wacc_clear(S.acc);
      for (int t = grank(g); t < T.ntiles; t += g.nblk) {
        const int x0 = (t % T.tiles_x) * TXo<Op>, y0 = (t / T.tiles_x) * TYo<Op>;
        fill_tile(op, tb, T, x0, y0, [&](const long long* c, VT (*v)[M]) {
#pragma unroll
          for (int r = 0; r < FQ; ++r)
#pragma unroll
            for (int m = 0; m < M; ++m) v[r][m] = (VT)ldcg(x + m * N + c[r]);
        });
        double rr = 0.0;
#pragma unroll
        for (int r = 0; r < CPTo<Op>; ++r) {
          const Cell k = tile_cell<Op>(T, x0, y0, r);
          if (!k.in) continue;
          VT ax[M];
          op.matvec(tb, k.lx, k.ly, k.c, ax);
          VT res[M];
#pragma unroll
          for (int m = 0; m < M; ++m) res[m] = (VT)(ldcg(b + m * N + k.c) - (double)ax[m]);
          op.precond(k.c, res);
#pragma unroll
          for (int m = 0; m < M; ++m) {
            const double rv = (double)res[m];
            Vp(0)[m * N + k.c] = (TS)rv;
            rr += rv * rv;
          }
        }
        wacc_add(S.acc, 0, rr);
        __syncthreads();
      }
      wacc_store(S.acc, 1, part() + (long long)grank(g) * NP);
      if (!grid_barrier(g.sync, g.nblk)) return GM_SYNC;
      grid_reduce(part(), g.nblk, 1, S.red, S.acc);
      ++phase;
      count(M, 2 * M + coef);
      S.gam[0] = sqrt(S.red[0]);
      if (outer == 0) tol_eff = g.tol * S.gam[0] + g.tol_abs;
      if (!isfinite(S.gam[0])) return GM_NONFINITE;
      if (S.gam[0] <= tol_eff) {
        if (lead) {
          g.st->gmres_iters += iters;
          g.st->last_residual = S.gam[0];
        }
        return GM_CONVERGED;
      }
      if (lead) g.st->gmres_restarts += 1;
      S.sigma[0] = 1.0 / S.gam[0];

      // ---- Av0 = M^-1 A V0 (unnormalised), H[0][0]
      wacc_clear(S.acc);
      for (int t = grank(g); t < T.ntiles; t += g.nblk) {
        const int x0 = (t % T.tiles_x) * TXo<Op>, y0 = (t / T.tiles_x) * TYo<Op>;
        fill_tile(op, tb, T, x0, y0, [&](const long long* c, VT (*v)[M]) {
#pragma unroll
          for (int r = 0; r < FQ; ++r)
#pragma unroll
            for (int m = 0; m < M; ++m) v[r][m] = (VT)ldv(Vp(0) + m * N + c[r]);
        });
        double va = 0.0;
#pragma unroll
        for (int r = 0; r < CPTo<Op>; ++r) {
          const Cell k = tile_cell<Op>(T, x0, y0, r);
          if (!k.in) continue;
          VT aw[M];
          op.matvec(tb, k.lx, k.ly, k.c, aw);
          op.precond(k.c, aw);
          const int o = (k.ly + Op::HALO) * TB::SX + k.lx + Op::HALO;
#pragma unroll
          for (int m = 0; m < M; ++m) {
            AVp(0)[m * N + k.c] = (TS)aw[m];
            va += (double)tb.s[m * TB::SN + o] * (double)aw[m];
          }
        }
        wacc_add(S.acc, 0, va);
        __syncthreads();
      }
      wacc_store(S.acc, 1, part() + (long long)grank(g) * NP);
      if (!grid_barrier(g.sync, g.nblk)) return GM_SYNC;
      grid_reduce(part(), g.nblk, 1, S.red, S.acc);
      ++phase;
      count(2 * M, coef);
      for (int r = threadIdx.x; r < (KCAP + 2) * (KCAP + 2); r += NT) (&S.H[0][0])[r] = 0.0;
      __syncthreads();
      if (threadIdx.x == 0) S.H[0][0] = S.sigma[0] * S.sigma[0] * S.red[0];
      __syncthreads();
    }

    int jend = -1;  // last Arnoldi index used in the update
    bool converged = false;
    for (int j = 0; j < kmax; ++j) {
      // ---- fused pass: w = Av_j - sum_i H[i][j] v_i ; V_{j+1} = w ; AV_{j+1} = M^-1 A w ; dots
      // (the combination is formed in FP64 whatever the storage type)
      wacc_clear(S.acc);
      const double sj = S.sigma[j];
      for (int t = grank(g); t < T.ntiles; t += g.nblk) {
        const int x0 = (t % T.tiles_x) * TXo<Op>, y0 = (t / T.tiles_x) * TYo<Op>;
        fill_tile(op, tb, T, x0, y0, [&](const long long* c, VT (*v)[M]) {
          const TS* AVj = AVp(j);
          double wv[FQ][M];
#pragma unroll
          for (int r = 0; r < FQ; ++r)
#pragma unroll
            for (int m = 0; m < M; ++m) wv[r][m] = sj * ldv(AVj + m * N + c[r]);
#pragma unroll 4
          for (int i = 0; i <= j; ++i) {
            const double hij = S.H[i][j], si = S.sigma[i];
            const TS* Vi = Vp(i);
#pragma unroll
            for (int r = 0; r < FQ; ++r)
#pragma unroll
              for (int m = 0; m < M; ++m) wv[r][m] = wv[r][m] - hij * (si * ldv(Vi + m * N + c[r]));
          }
#pragma unroll
          for (int r = 0; r < FQ; ++r)
#pragma unroll
            for (int m = 0; m < M; ++m) v[r][m] = (VT)wv[r][m];
        });
        VT aw[CPTo<Op>][M], wc[CPTo<Op>][M];
        long long cc[CPTo<Op>];
        bool in[CPTo<Op>];
#pragma unroll
        for (int r = 0; r < CPTo<Op>; ++r) {
          const Cell k = tile_cell<Op>(T, x0, y0, r);
          cc[r] = k.c;
          in[r] = k.in;
          if (k.in) {
            op.matvec(tb, k.lx, k.ly, k.c, aw[r]);
            op.precond(k.c, aw[r]);
            const int o = (k.ly + Op::HALO) * TB::SX + k.lx + Op::HALO;
#pragma unroll
            for (int m = 0; m < M; ++m) {
              wc[r][m] = tb.s[m * TB::SN + o];
              Vp(j + 1)[m * N + k.c] = (TS)wc[r][m];
              AVp(j + 1)[m * N + k.c] = (TS)aw[r][m];
            }
          } else {
#pragma unroll
            for (int m = 0; m < M; ++m) aw[r][m] = wc[r][m] = VT(0);
          }
        }
        // slots: v_i.Aw -> i (i <= j), w.Aw -> j+1, w.w -> j+2; eight, then four basis vectors
        // at a time (independent loads in flight)
        int i = 0;
        for (; i + 7 <= j; i += 8) {
          double d[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
          for (int r = 0; r < CPTo<Op>; ++r)
            if (in[r]) {
#pragma unroll
              for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int m = 0; m < M; ++m) d[u] += ldv(Vp(i + u) + m * N + cc[r]) * (double)aw[r][m];
            }
          wacc_add4(S.acc, i, *reinterpret_cast<double(*)[4]>(&d[0]));
          wacc_add4(S.acc, i + 4, *reinterpret_cast<double(*)[4]>(&d[4]));
        }
        for (; i + 3 <= j; i += 4) {
          double d[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
          for (int r = 0; r < CPTo<Op>; ++r)
            if (in[r]) {
#pragma unroll
              for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int m = 0; m < M; ++m) d[u] += ldv(Vp(i + u) + m * N + cc[r]) * (double)aw[r][m];
            }
          wacc_add4(S.acc, i, d);
        }
        for (; i <= j; ++i) {
          double d = 0.0;
#pragma unroll
          for (int r = 0; r < CPTo<Op>; ++r)
            if (in[r]) {
#pragma unroll
              for (int m = 0; m < M; ++m) d += ldv(Vp(i) + m * N + cc[r]) * (double)aw[r][m];
            }
          wacc_add(S.acc, i, d);
        }
        double wa = 0.0, ww = 0.0;
#pragma unroll
        for (int r = 0; r < CPTo<Op>; ++r)
#pragma unroll
          for (int m = 0; m < M; ++m) {
            wa += (double)wc[r][m] * (double)aw[r][m];
            ww += (double)wc[r][m] * (double)wc[r][m];
          }
        wacc_add(S.acc, j + 1, wa);
        wacc_add(S.acc, j + 2, ww);
        __syncthreads();
      }
      wacc_store(S.acc, j + 3, part() + (long long)grank(g) * NP);
      if (!grid_barrier(g.sync, g.nblk)) return GM_SYNC;
      grid_reduce(part(), g.nblk, j + 3, S.red, S.acc);
      ++phase;
      ++iters;
      count((j + 4) * M, coef);
      if (threadIdx.x == 0) {
        // H[j+1][j] = |w|; Givens on column j (implicit_operators.cpp:857-873)
        const double beta_w = sqrt(S.red[j + 2]);
        S.H[j + 1][j] = beta_w;
        for (int i = 0; i < j; i++) {
          double t1 = S.cs[i + 1] * S.H[i][j] + S.sn[i + 1] * S.H[i + 1][j];
          double t2 = S.sn[i + 1] * S.H[i][j] - S.cs[i + 1] * S.H[i + 1][j];
          S.H[i][j] = t1;
          S.H[i + 1][j] = t2;
        }
        double beta = sqrt(S.H[j][j] * S.H[j][j] + S.H[j + 1][j] * S.H[j + 1][j]);
        S.sn[j + 1] = S.H[j + 1][j] / beta;
        S.cs[j + 1] = S.H[j][j] / beta;
        S.H[j][j] = beta;
        S.gam[j + 1] = S.sn[j + 1] * S.gam[j];
        S.gam[j] = S.cs[j + 1] * S.gam[j];
        // column j+1 of H from the fused dots: v_i . Av_{j+1}
        const double sw = 1.0 / beta_w;
        S.sigma[j + 1] = sw;
        if (j + 1 < KCAP + 1) {
          for (int i = 0; i <= j; ++i) S.H[i][j + 1] = S.sigma[i] * S.red[i] * sw;
          S.H[j + 1][j + 1] = sw * sw * S.red[j + 1];
        }
      }
      __syncthreads();
      if (!isfinite(S.gam[j + 1])) return GM_NONFINITE;
      if (!(S.gam[j + 1] > tol_eff)) {
        jend = j;
        converged = true;
        break;
      }
      jend = j;
    }
    // ---- back substitution and x += sum alpha_i v_i (implicit_operators.cpp:882-891, 900-910)
    if (threadIdx.x == 0) {
      for (int i = jend; i >= 0; i--) {
        S.alpha[i] = S.gam[i];
        for (int k = i + 1; k <= jend; k++) S.alpha[i] -= S.H[i][k] * S.alpha[k];
        S.alpha[i] /= S.H[i][i];
      }
    }
    __syncthreads();
    if (defer && (converged || last_cycle)) {
      if (threadIdx.x == 0) S.nalpha = jend + 1;
      __syncthreads();
      if (lead) {
        g.st->gmres_iters += iters;
        g.st->last_residual = S.gam[jend + 1];
      }
      return converged ? GM_CONVERGED : GM_MAXIT;
    }
    for (long long c = grank(g) * (long long)NT + threadIdx.x; c < N; c += (long long)g.nblk * NT) {
#pragma unroll
      for (int m = 0; m < M; ++m) {
        double xv = from_zero ? 0.0 : ldcg(x + m * N + c);
        for (int i = 0; i <= jend; ++i) xv = xv + S.alpha[i] * (S.sigma[i] * ldv(Vp(i) + m * N + c));
        x[m * N + c] = xv;
      }
    }
    x_written = true;
    if (!grid_barrier(g.sync, g.nblk)) return GM_SYNC;
    count((jend + 1) * M, (from_zero ? 1 : 2) * M);
    if (converged) {
      if (threadIdx.x == 0 && grank(g) == 0) {
        g.st->gmres_iters += iters;
        g.st->last_residual = S.gam[jend + 1];
      }
      return GM_CONVERGED;
    }
  }
  if (threadIdx.x == 0 && grank(g) == 0) g.st->gmres_iters += iters;
  return GM_MAXIT;
}

// the worst status of a solve, recorded once (by the solve's first CTA)
template <class W>
__device__ __forceinline__ void record_status(const W& g, int code) {
  DevStats* st = g.st;
  if (threadIdx.x == 0 && grank(g) == 0) {
    int s = IMEX_OK;
    if (code == GM_MAXIT) s = IMEX_GMRES_MAXIT;
    else if (code == GM_NONFINITE) s = IMEX_NONFINITE;
    else if (code == GM_SYNC) s = IMEX_ERR_SYNC;
    if (s != IMEX_OK) atomicMax(&st->status, s);
  }
}

// shared memory of one solver CTA (dynamic, opted in above 48 KB)
template <class Op>
struct SolveSmem {
  GmresShared S;
  TileBuf<Op> tb;
};

template <class Op>
__device__ __forceinline__ void gmres_solve(Op op, GmresWork g, double* x, const double* b) {
  extern __shared__ __align__(16) unsigned char dsm[];
  SolveSmem<Op>& sm = *reinterpret_cast<SolveSmem<Op>*>(dsm);
  GmresShared& S = sm.S;
  TileBuf<Op>& tb = sm.tb;
  unsigned phase = 0;
  op.bind();
  if (threadIdx.x == 0 && grank(g) == 0) g.st->gmres_solves += 1;
  bool written = false;
  int code = gmres_device(op, g, x, b, S, tb, phase, false, false, written);
  record_status(g, code);
}
template <class Op>
__global__ void __launch_bounds__(NT, Op::MIN_BLOCKS) k_gmres(Op op, GmresWork g, double* x, const double* b) {
  gmres_solve(op, g, x, b);
}

// Batched solves: one cooperative launch runs many independent solves (the members of an
// ensemble).  Solve m owns the contiguous CTAs [g.first, g.first + g.nblk) of the launch,
// with its own barrier state, partial sums and statistics, so solves never wait on one
// another; cta_job maps each CTA to its solve.
template <class Op>
struct GmresJob {
  Op op;
  GmresWork g;
  double* x;
  const double* b;
};
template <class Op>
__global__ void __launch_bounds__(NT, Op::MIN_BLOCKS) k_gmres_jobs(const GmresJob<Op>* jobs, const int* cta_job) {
  const GmresJob<Op>& j = jobs[cta_job[blockIdx.x]];
  gmres_solve(j.op, j.g, j.x, j.b);
}

// ------------------------------------------------------------------ mixed-precision GMRES
// The mixed form of GMRES_Solver: FP64 iterative refinement around FP32 inner solves.
//   each sweep, one FP64 pass: x <- x + (pending inner update), s = b - A x and |M^-1 s|
//     in FP64 arithmetic with FP64 coefficients; stop at |M^-1 s| <= GMREStol |r_0| + GMREStol,
//     the stopping rule of the plain form, or when the FP64 residual has reached its rounding
//     floor: an inner cycle met its tolerance and yet the true residual fell by less than half,
//     or two sweeps in a row fell by less than half (the plain form tests the recursive GMRES
//     estimate, which keeps falling below that floor);
//   then one FP32 inner GMRES cycle on M^-1 A d = M^-1 s from d = 0 (operator and preconditioner
//     in FP32, basis stored in FP32, Gram-Schmidt dots and the Hessenberg solve in FP64), stopped
//     at a relative residual of g.tol or after g.kmax steps; its update sum_i alpha_i v_i is
//     added to x inside the next FP64 pass.
// x is double buffered between x and xalt (the FP64 pass reads the old iterate on the tile
// halo); the result ends in x.
template <class Op64>
struct MixedSmem {
  using Op32 = decltype(Op64().template as<float>());
  GmresShared S;
  union {
    TileBuf<Op64> d;
    TileBuf<Op32> f;
  } tb;
};

template <class Op64>
__device__ __forceinline__ void mixed_solve(Op64 op, GmresWorkT<float> g, double* x, double* xalt, double* sres,
                                            const double* b, int max_sweeps, double tol) {
  using Op32 = typename MixedSmem<Op64>::Op32;
  using TB = TileBuf<Op64>;
  constexpr int M = Op64::M, FQ = FillQ<Op64>;
  extern __shared__ __align__(16) unsigned char dsm[];
  MixedSmem<Op64>& sm = *reinterpret_cast<MixedSmem<Op64>*>(dsm);
  GmresShared& S = sm.S;
  op.bind();
  const Op32 op32 = op.template as<float>();
  const Tiling& T = g.T;
  const long long N = T.N;
  unsigned phase = 0;
  auto part = [&]() { return g.partial + (long long)(phase & 1) * g.nblk * NP; };
  const bool lead = threadIdx.x == 0 && grank(g) == 0;
  const int coef = Op64::COEF + (op_uses_vdiag(op) ? 1 : 0);
  if (lead) g.st->gmres_solves += 1;
  double* x_cur = x;
  double* x_nxt = xalt;
  bool pending = false, inner_ok = false;
  int stalls = 0;
  double tol_eff = 0.0, prev = INFINITY;
  int code = GM_MAXIT;
  for (int sweep = 0;; ++sweep) {
    // ---- FP64: x += pending update; s = b - A x; |M^-1 s|^2
    wacc_clear(S.acc);
    for (int t = grank(g); t < T.ntiles; t += g.nblk) {
      const int x0 = (t % T.tiles_x) * TXo<Op64>, y0 = (t / T.tiles_x) * TYo<Op64>;
      fill_tile(op, sm.tb.d, T, x0, y0, [&](const long long* c, double (*v)[M]) {
#pragma unroll
        for (int r = 0; r < FQ; ++r)
#pragma unroll
          for (int m = 0; m < M; ++m) {
            double xv = ldcg(x_cur + m * N + c[r]);
            if (pending)
              for (int i = 0; i < S.nalpha; ++i)
                xv = xv + S.alpha[i] * (S.sigma[i] * ldv(g.V + (long long)i * M * N + m * N + c[r]));
            v[r][m] = xv;
          }
      });
      double rr = 0.0;
#pragma unroll
      for (int r = 0; r < CPTo<Op64>; ++r) {
        const Cell k = tile_cell<Op64>(T, x0, y0, r);
        if (!k.in) continue;
        double ax[M], res[M];
        op.matvec(sm.tb.d, k.lx, k.ly, k.c, ax);
        const int o = (k.ly + Op64::HALO) * TB::SX + k.lx + Op64::HALO;
#pragma unroll
        for (int m = 0; m < M; ++m) {
          if (pending) x_nxt[m * N + k.c] = sm.tb.d.s[m * TB::SN + o];
          res[m] = ldcg(b + m * N + k.c) - ax[m];
          sres[m * N + k.c] = res[m];
        }
        op.precond(k.c, res);
#pragma unroll
        for (int m = 0; m < M; ++m) rr += res[m] * res[m];
      }
      wacc_add(S.acc, 0, rr);
      __syncthreads();
    }
    wacc_store(S.acc, 1, part() + (long long)grank(g) * NP);
    if (!grid_barrier(g.sync, g.nblk)) {
      record_status(g, GM_SYNC);
      return;
    }
    grid_reduce(part(), g.nblk, 1, S.red, S.acc);
    ++phase;
    if (lead)
      g.st->alg_bytes[g.fam] += ((double)((pending ? 3 : 2) * M + M + coef) * 8.0 +
                                 (pending ? (double)S.nalpha * M * sizeof(float) : 0.0)) * (double)N;
    if (pending) {
      double* t = x_cur;
      x_cur = x_nxt;
      x_nxt = t;
      pending = false;
    }
    const double res = sqrt(S.red[0]);
    if (sweep == 0) tol_eff = tol * res + tol;
    if (!isfinite(res)) {
      code = GM_NONFINITE;
      break;
    }
    if (lead) g.st->last_residual = res;
    stalls = res > 0.5 * prev ? stalls + 1 : 0;
    if (res <= tol_eff || (inner_ok && res > 0.5 * prev) || stalls >= 2) {
      code = GM_CONVERGED;
      break;
    }
    prev = res;
    if (sweep >= max_sweeps) break;
    // ---- FP32 inner cycle on M^-1 A d = M^-1 s, update deferred
    if (lead) g.st->refine_sweeps += 1;
    bool written = false;
    int c2 = gmres_device(op32, g, x_nxt, sres, S, sm.tb.f, phase, true, true, written);
    if (c2 == GM_SYNC || c2 == GM_NONFINITE) {
      record_status(g, c2);
      return;
    }
    inner_ok = c2 == GM_CONVERGED;
    pending = true;
  }
  // the result ends in x
  if (x_cur != x)
    for (long long c = grank(g) * (long long)NT + threadIdx.x; c < (long long)M * N; c += (long long)g.nblk * NT)
      x[c] = ldcg(x_cur + c);
  if (code != GM_CONVERGED) record_status(g, code);
}
template <class Op64>
__global__ void __launch_bounds__(NT, Op64::MIN_BLOCKS)
    k_gmres_mixed(Op64 op, GmresWorkT<float> g, double* x, double* xalt, double* sres, const double* b,
                  int max_sweeps, double tol) {
  mixed_solve(op, g, x, xalt, sres, b, max_sweeps, tol);
}
template <class Op64>
struct MixedJob {
  Op64 op;
  GmresWorkT<float> g;
  double *x, *xalt, *sres;
  const double* b;
  int max_sweeps;
  double tol;
};
template <class Op64>
__global__ void __launch_bounds__(NT, Op64::MIN_BLOCKS) k_gmres_mixed_jobs(const MixedJob<Op64>* jobs,
                                                                          const int* cta_job) {
  const MixedJob<Op64>& j = jobs[cta_job[blockIdx.x]];
  mixed_solve(j.op, j.g, j.x, j.xalt, j.sres, j.b, j.max_sweeps, j.tol);
}

// ------------------------------------------------------------------ nested Newton
// Pressure_NestedNewton (implicit_operators.cpp:625-738) on the device.
struct NewtonArgs {
  double *p, *pf, *g, *dp, *vdiag;
  const double* b;
  DevScalars* sc;
  const unsigned long long* bkeys;  // min b / max V keys from k_pressure_rhs, or null: reduce here
};

// Shared memory of the nested Newton: the FP64 tile of the residual passes and the
// tile of the Jacobian solves (FP64, or FP32 in the mixed form) share one buffer.
template <class TS>
struct NewtonSmem {
  GmresShared S;
  union {
    TileBuf<PressureOp> l;
    TileBuf<PressureOpT<TS>> j;
  } tb;
};

// The Jacobian solves store their Krylov basis as TS and apply the operator in TS
// arithmetic (double: the plain form; float: the mixed form).  The residual, the
// Newton convergence test and the iterate stay FP64 in both.  Only the floored or
// Redlich-Kwong case comes here; the linear case is a plain GMRES launch.
template <class TS>
__device__ __forceinline__ void newton_solve(PressureOp op, GmresWorkT<TS> gw, NewtonArgs na) {
  op.bind();
  extern __shared__ __align__(16) unsigned char dsm[];
  NewtonSmem<TS>& sm = *reinterpret_cast<NewtonSmem<TS>*>(dsm);
  GmresShared& S = sm.S;
  TileBuf<PressureOp>& tb = sm.tb.l;
  using TB = TileBuf<PressureOp>;
  const DevParams& P = op.P;
  const Tiling& T = gw.T;
  const long long N = T.N;
  unsigned phase = 0;
  auto part = [&]() { return gw.partial + (long long)(phase & 1) * gw.nblk * NP; };
  const bool lead = threadIdx.x == 0 && grank(gw) == 0;

  // ---- Cor. 1 slope Mbig (implicit_operators.cpp:670-686)
  double Mbig = na.sc->Mbig;
  if (P.floor_on && na.bkeys) {
    // min b and max V(p_floor, rho) came with the right-hand side (k_pressure_rhs)
    const unsigned long long kb = na.bkeys[0], kv = ~na.bkeys[1];
    const double bmin = kb == ~0ull ? INFINITY : dkey_value(kb);
    double Vpe = P.p_floor / (P.gamma - 1.0);
    if (P.eos_type != IMEX_IDEAL_GAS && kv != 0ull && dkey_value(kv) > Vpe) Vpe = dkey_value(kv);
    double q = Vpe - bmin;
    double M_cor = ((0.0 < q) ? q : 0.0) / ((1.0 - P.theta) * P.p_floor);
    double M_base = P.Mbig_fac / (P.gamma - 1.0);
    Mbig = (M_base < M_cor) ? M_cor : M_base;
    if (lead) na.sc->Mbig = Mbig;
  } else if (P.floor_on) {
    double mn = INFINITY, vpe = -INFINITY;
    for (long long c = grank(gw) * (long long)NT + threadIdx.x; c < N; c += (long long)gw.nblk * NT) {
      mn = fmin(mn, na.b[c]);
      if (P.eos_type != IMEX_IDEAL_GAS) {
        double v = Vbase(P, P.p_floor, __ldg(op.rho + c));
        if (isfinite(v)) vpe = fmax(vpe, v);
      }
    }
    double a2[2] = {mn, vpe};
    // block min / max via shared memory
    __shared__ double shm[2][NT / 32];
    for (int o = 16; o > 0; o >>= 1) {
      a2[0] = fmin(a2[0], __shfl_xor_sync(0xffffffffu, a2[0], o));
      a2[1] = fmax(a2[1], __shfl_xor_sync(0xffffffffu, a2[1], o));
    }
    if ((threadIdx.x & 31) == 0) {
      shm[0][threadIdx.x >> 5] = a2[0];
      shm[1][threadIdx.x >> 5] = a2[1];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double m0 = INFINITY, m1 = -INFINITY;
      for (int w = 0; w < NT / 32; ++w) {
        m0 = fmin(m0, shm[0][w]);
        m1 = fmax(m1, shm[1][w]);
      }
      part()[(long long)grank(gw) * NP + 0] = m0;
      part()[(long long)grank(gw) * NP + 1] = m1;
    }
    if (!grid_barrier(gw.sync, gw.nblk)) {
      record_status(gw, GM_SYNC);
      return;
    }
    grid_reduce(part(), gw.nblk, 2, S.red, S.acc, RED_MIN | (RED_MAX << 2));
    ++phase;
    double bmin = S.red[0];
    double Vpe = P.p_floor / (P.gamma - 1.0);
    if (P.eos_type != IMEX_IDEAL_GAS && S.red[1] > Vpe) Vpe = S.red[1];
    double q = Vpe - bmin;
    double M_cor = ((0.0 < q) ? q : 0.0) / ((1.0 - P.theta) * P.p_floor);
    double M_base = P.Mbig_fac / (P.gamma - 1.0);
    Mbig = (M_base < M_cor) ? M_cor : M_base;
    if (lead) {
      na.sc->Mbig = Mbig;
      gw.st->alg_bytes[gw.fam] += (P.eos_type != IMEX_IDEAL_GAS ? 2.0 : 1.0) * 8.0 * (double)N;
    }
  }
  PressureOp L = op;
  L.jac = 0;
  PressureOpT<TS> J = op.as<TS>();
  J.jac = 1;
  J.vdiag = na.vdiag;
  const double a = op.a;
  double res0 = -1.0;
  // The Newton iterate pf is double buffered between p (which holds the initial guess) and
  // the pf plane: each residual pass reads pf_cur at the tile halo and writes the updated
  // iterate to pf_nxt.  The Jacobian GMRES runs in deferred mode, so its update
  // dp = sum_i alpha_i v_i (+ dp when an earlier restart cycle wrote it) is added to pf
  // inside the next residual pass instead of in two passes of its own.
  double* pf_cur = na.p;
  double* pf_nxt = na.pf;
  bool pending = false;  // a GMRES update waits to be added to pf
  bool dp_live = false;  // dp holds the part of that update written by restart cycles
  auto pf_update = [&](long long c) {
    double d = dp_live ? ldcg(na.dp + c) : 0.0;
    for (int i = 0; i < S.nalpha; ++i) d = d + S.alpha[i] * (S.sigma[i] * ldv(gw.V + (long long)i * N + c));
    return ldcg(pf_cur + c) + d;
  };
  int it;
  for (it = 0; it < P.Pnewton_max; it++) {
    // ---- pf += pending update; residual g = L pf - a pf + V_mod(pf) - b -> na.g = -g; vdiag = V_slope(pf)
    wacc_clear(S.acc);
    for (int t = grank(gw); t < T.ntiles; t += gw.nblk) {
      const int x0 = (t % T.tiles_x) * TXo<PressureOp>, y0 = (t / T.tiles_x) * TYo<PressureOp>;
      fill_tile(L, tb, T, x0, y0, [&](const long long* c, double (*v)[1]) {
        if (pending) {
#pragma unroll
          for (int r = 0; r < FillQ<PressureOp>; ++r) v[r][0] = pf_update(c[r]);
        } else {
#pragma unroll
          for (int r = 0; r < FillQ<PressureOp>; ++r) v[r][0] = ldcg(pf_cur + c[r]);
        }
      });
      double gg = 0.0;
#pragma unroll
      for (int r = 0; r < CPTo<PressureOp>; ++r) {
        const Cell k = tile_cell<PressureOp>(T, x0, y0, r);
        if (!k.in) continue;
        double lp[1];
        L.matvec(tb, k.lx, k.ly, k.c, lp);
        const double pfc = tb.s[(k.ly + 1) * TB::SX + k.lx + 1];
        if (pending) pf_nxt[k.c] = pfc;
        const double rc = __ldg(op.rho + k.c);
        const double gv = lp[0] - a * pfc + V_mod(P, Mbig, pfc, rc) - na.b[k.c];
        gg += gv * gv;
        na.g[k.c] = -gv;
        na.vdiag[k.c] = V_slope(P, Mbig, pfc, rc);
      }
      wacc_add(S.acc, 0, gg);
      __syncthreads();
    }
    wacc_store(S.acc, 1, part() + (long long)grank(gw) * NP);
    if (!grid_barrier(gw.sync, gw.nblk)) {
      record_status(gw, GM_SYNC);
      return;
    }
    grid_reduce(part(), gw.nblk, 1, S.red, S.acc);
    ++phase;
    if (lead)
      gw.st->alg_bytes[gw.fam] +=
          ((double)(PressureOp::COEF + 4 + (pending ? 1 + (dp_live ? 1 : 0) : 0)) * 8.0 +
           (pending ? (double)S.nalpha * sizeof(TS) : 0.0)) * (double)N;
    if (pending) {
      double* t = pf_cur;
      pf_cur = pf_nxt;
      pf_nxt = t;
      pending = false;
    }
    const double res = sqrt(S.red[0]);
    if (it == 0) res0 = res;
    if (!isfinite(res)) {
      record_status(gw, GM_NONFINITE);
      break;
    }
    if (res < P.Pnewton_tol * res0 + P.Pnewton_tol) break;
    // ---- Jacobian solve J dp = -g (GMRES with precP), from dp = 0, update deferred
    if (lead) {
      gw.st->gmres_solves += 1;
      gw.st->newton_iters += 1;
    }
    int code = gmres_device(J, gw, na.dp, na.g, S, sm.tb.j, phase, true, true, dp_live);
    if (code != GM_CONVERGED) {
      record_status(gw, code);
      if (code == GM_SYNC || code == GM_NONFINITE) return;
    }
    pending = true;
  }
  if (it == P.Pnewton_max && lead) atomicMax(&gw.st->status, (int)IMEX_NEWTON_MAXIT);
  if (lead)
    gw.st->alg_bytes[gw.fam] += ((double)(2 + (pending && dp_live ? 1 : 0)) * 8.0 +
                                 (pending ? (double)S.nalpha * sizeof(TS) : 0.0)) * (double)N;
  // ---- p = pf (+ an update still pending after Pnewton_max), floored-cell count and min p
  // (implicit_operators.cpp:722-737)
  double st2[2] = {0.0, INFINITY};
  for (long long c = grank(gw) * (long long)NT + threadIdx.x; c < N; c += (long long)gw.nblk * NT) {
    const double pv = pending ? pf_update(c) : ldcg(pf_cur + c);
    na.p[c] = pv;
    if (pv < P.p_floor) st2[0] += 1.0;
    st2[1] = fmin(st2[1], pv);
  }
  if (P.floor_on) {
    __shared__ double sh2[2][NT / 32];
    for (int o = 16; o > 0; o >>= 1) {
      st2[0] += __shfl_xor_sync(0xffffffffu, st2[0], o);
      st2[1] = fmin(st2[1], __shfl_xor_sync(0xffffffffu, st2[1], o));
    }
    if ((threadIdx.x & 31) == 0) {
      sh2[0][threadIdx.x >> 5] = st2[0];
      sh2[1][threadIdx.x >> 5] = st2[1];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double s0 = 0.0, s1 = INFINITY;
      for (int w = 0; w < NT / 32; ++w) {
        s0 += sh2[0][w];
        s1 = fmin(s1, sh2[1][w]);
      }
      part()[(long long)grank(gw) * NP + 0] = s0;
      part()[(long long)grank(gw) * NP + 1] = s1;
    }
    if (!grid_barrier(gw.sync, gw.nblk)) {
      record_status(gw, GM_SYNC);
      return;
    }
    grid_reduce(part(), gw.nblk, 2, S.red, S.acc, RED_SUM | (RED_MIN << 2));
    if (lead) {
      const double nf = S.red[0], pmin = S.red[1];
      if ((int)nf > gw.st->max_floored) gw.st->max_floored = (int)nf;
      if (pmin < gw.st->min_p) gw.st->min_p = pmin;
      if (pmin < P.theta * P.p_floor - 1e-14) atomicMax(&gw.st->status, (int)IMEX_POSITIVITY);
    }
  }
}

// kRK = false: the ideal-gas instance.  Its EOS branches fold at compile time, so it carries
// none of the Redlich-Kwong Newton iterations and its code stays small (this persistent
// kernel is large enough for instruction fetch to stall it).
// kMinB: CTAs per SM the registers are sized for.  Three (80 registers, a few hundred bytes
// spilled) hide more load latency once a solve's planes no longer fit in the L2; two keep
// the spills away while they do (newton_launch chooses by grid size).
template <class TS, bool kRK = true, int kMinB = 2>
__global__ void __launch_bounds__(NT, kMinB) k_nested_newton(PressureOp op, GmresWorkT<TS> gw, NewtonArgs na) {
  if (!kRK) op.P.eos_type = IMEX_IDEAL_GAS;
  newton_solve(op, gw, na);
}
template <class TS>
struct NewtonJob {
  PressureOp op;
  GmresWorkT<TS> gw;
  NewtonArgs na;
};
// kRK as for k_nested_newton; three CTAs per SM (an ensemble's members together outgrow the L2)
template <class TS, bool kRK = true>
__global__ void __launch_bounds__(NT, 3) k_nested_newton_jobs(const NewtonJob<TS>* jobs, const int* cta_job) {
  const NewtonJob<TS>& j = jobs[cta_job[blockIdx.x]];
  PressureOp op = j.op;
  if (!kRK) op.P.eos_type = IMEX_IDEAL_GAS;
  newton_solve(op, j.gw, j.na);
}

// the barrier states of the solves of one batched launch start at zero
__global__ void k_reset_syncs(SyncState* const* syncs, int n, long long limit) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    syncs[i]->count = 0;
    syncs[i]->abort = 0;
    syncs[i]->wait_cycles = limit;
  }
}

// ------------------------------------------------------------------ elementwise kernels
constexpr int kThreads = 256;
inline int blocks_for(long long n) { return (int)((n + kThreads - 1) / kThreads); }

// enthalpy ratio h(Qe) rho_e / rho, V slope at p(Qe), rho v* snapshot (imex_subsystems.cpp:92-147)
template <bool kOpen>
struct k_pressure_coeffs {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams Pin, const double* __restrict__ Qe, const double* __restrict__ ucon,
                                    const double* __restrict__ hQe, const double* __restrict__ pe,
                                    double* __restrict__ hh, double* __restrict__ vscale, double* __restrict__ rv,
                                    unsigned long long* __restrict__ bkeys) {
    const DevParams P = bc_params<kOpen>(Pin);
    const long long N = P.N;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n < 4) bkeys[n] = ~0ull;  // the identities of the min keys k_pressure_rhs forms next
    if (n >= N) return;
    const double r = ucon[n], hq = hQe[n], q = Qe[n], pn = pe[n];
    const double m1 = ucon[N + n], m2 = ucon[2 * N + n], m3 = ucon[3 * N + n];
    rv[n] = m1;
    rv[N + n] = m2;
    rv[2 * N + n] = m3;
    hh[n] = hq * q / r;
    vscale[n] = Vbase_slope(P, pn, r);
  }
};
// Jacobi diagonal Tdiag (implicit_operators.cpp:631-649)
template <bool kOpen>
struct k_pressure_tdiag {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams Pin, const DevScalars* __restrict__ sc, const double* __restrict__ hh,
                                   double* __restrict__ tdiag) {
    const DevParams P = bc_params<kOpen>(Pin);
    const double h = sc->h;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= P.N) return;
    int i, j;
    cell_of(P, n, i, j);
    const double h00 = hh[n], hp0 = hh[cid(P, i + 1, j)], hm0 = hh[cid(P, i - 1, j)], h0p = hh[cid(P, i, j + 1)],
                 h0m = hh[cid(P, i, j - 1)];
    tdiag[n] = h * h * ((0.5 * (hp0 + h00) + 0.5 * (hm0 + h00)) / (P.dx * P.dx) +
                        (0.5 * (h0p + h00) + 0.5 * (h0m + h00)) / (P.dy * P.dy));
  }
};
// pressure RHS b (imex_subsystems.cpp:123-169 first, 226-269 second); kin = momentum used in
// the kinetic term, rv = rho v* used in the enthalpy-flux divergence; p0 = initial guess.
template <bool kOpen>
struct k_pressure_rhs {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams Pin, const DevScalars* __restrict__ sc, const double* __restrict__ ucon,
                                 const double* __restrict__ hh, const double* __restrict__ rv,
                                 const double* __restrict__ kin, double* __restrict__ b,
                                 const double* __restrict__ p0src, double* __restrict__ p0,
                                 unsigned long long* __restrict__ bkeys) {
    const DevParams P = bc_params<kOpen>(Pin);
    const long long N = P.N;
    const double h = sc->h;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    unsigned long long kb = ~0ull, kv = ~0ull;  // identities of min
    if (n < N) {
      long long nb[9];
      neighbours(P, n, nb);
      const double* arr[4] = {ucon, hh, rv, kin};
      auto ld = [&](int a, int k, long long m) { return arr[a][k * N + m]; };
      double out[1];
      pressure_rhs_cell<double>(P, h, nb, ld, out);
      b[n] = out[0];
      if (p0) p0[n] = p0src[n];
      if (out[0] == out[0]) kb = dkey(out[0]);
      if (P.floor_on && P.eos_type != IMEX_IDEAL_GAS) {
        const double v = Vbase(P, P.p_floor, ucon[n]);
        if (isfinite(v)) kv = ~dkey(v);
      }
    }
    // the nested Newton's Cor.1 inputs (implicit_operators.cpp:670-686): min b and max V(p_floor,
    // rho), as exact order-key minima, so that the solve needs no reduction pass of its own
    if (bkeys) {
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long ob = __shfl_xor_sync(0xffffffffu, kb, o), ov = __shfl_xor_sync(0xffffffffu, kv, o);
        kb = ob < kb ? ob : kb;
        kv = ov < kv ? ov : kv;
      }
      __shared__ unsigned long long sk[2][kThreads / 32];
      if ((threadIdx.x & 31) == 0) {
        sk[0][threadIdx.x >> 5] = kb;
        sk[1][threadIdx.x >> 5] = kv;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
          kb = sk[0][w] < kb ? sk[0][w] : kb;
          kv = sk[1][w] < kv ? sk[1][w] : kv;
        }
        if (kb < *(volatile unsigned long long*)&bkeys[0]) atomicMin(&bkeys[0], kb);
        if (kv < *(volatile unsigned long long*)&bkeys[1]) atomicMin(&bkeys[1], kv);
      }
    }
  }
};
// momentum correction rho v = rho v* - h grad p (imex_subsystems.cpp:186-215)
struct k_momentum {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const DevScalars* __restrict__ sc, const double* __restrict__ p,
                             const double* __restrict__ rv, double* __restrict__ ucon) {
    const long long N = P.N;
    const double h = sc->h;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    long long nb[9];
    neighbours(P, n, nb);
    const double* arr[2] = {p, rv};
    auto ld = [&](int a, int k, long long m) { return arr[a][k * N + m]; };
    double out[2];
    momentum_cell<double>(P, h, nb, ld, out);
    ucon[N + n] = out[0];
    ucon[2 * N + n] = out[1];
  }
};
// E = V(p) + KE + ME (DefinitionofU, imex_subsystems.cpp:286-302)
struct k_energy_define {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const double* __restrict__ p, double* __restrict__ ucon) {
    const long long N = P.N;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    long long nb[9];
    nb[NB_C] = n;
    const double* arr[2] = {p, ucon};
    auto ld = [&](int a, int k, long long m) { return arr[a][k * N + m]; };
    double out[1];
    energy_define_cell<double>(P, nb, ld, out);
    ucon[4 * N + n] = out[0];
  }
};

// E -= h div(h_e rho v) (ConservationofU, imex_subsystems.cpp:303-392).  Reads only the
// density and momentum planes of the neighbours, so E is updated in place.
struct k_energy_conservation {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const DevScalars* __restrict__ sc, const double* __restrict__ p,
                                        double* __restrict__ ucon) {
    const long long N = P.N;
    const double h = sc->h;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    long long nb[9];
    neighbours(P, n, nb);
    const double* arr[2] = {p, ucon};
    auto ld = [&](int a, int k, long long m) { return arr[a][k * N + m]; };
    double out[1];
    energy_conservation_cell<double>(P, h, nb, ld, out);
    ucon[4 * N + n] = out[0];
  }
};

// total-enthalpy ratio hh = caltotalenthalpy(Qe) rho_e / rho (imex_subsystems.cpp:442-446)
struct k_energy_coeffs {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const double* __restrict__ Qe, const double* __restrict__ ucon,
                                  double* __restrict__ hh) {
    const long long N = P.N;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    double c[8];
  #pragma unroll
    for (int k = 0; k < 8; ++k) c[k] = Qe[k * N + n];
    hh[n] = caltotalenthalpy(P, c) * c[0] / ucon[n];
  }
};
// right-hand side b = U* dx dy (imex_subsystems.cpp:448-452) and the Jacobi scale diag dx dy
// of precE (imex_subsystems.cpp:499-503); the initial guess is E of u_con (solved in place)
struct k_energy_rhs {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const DevScalars* __restrict__ sc, const double* __restrict__ ucon,
                               const double* __restrict__ hh, double* __restrict__ b, double* __restrict__ tdiag) {
    const long long N = P.N;
    const double h = sc->h;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    int i, j;
    cell_of(P, n, i, j);
    const long long e = cid(P, i + 1, j), w = cid(P, i - 1, j), no = cid(P, i, j + 1), s = cid(P, i, j - 1);
    const double h00 = hh[n], hp0 = hh[e], hm0 = hh[w], h0p = hh[no], h0m = hh[s];
    const double U_star = ucon[4 * N + n] - 0.5 * h / P.dx * (hp0 * ucon[N + e] - hm0 * ucon[N + w]) -
                          0.5 * h / P.dy * (h0p * ucon[2 * N + no] - h0m * ucon[2 * N + s]);
    b[n] = U_star * P.dx * P.dy;
    const double hhp_x = 0.5 * (h00 + hp0), hhm_x = 0.5 * (h00 + hm0);
    const double hhp_y = 0.5 * (h00 + h0p), hhm_y = 0.5 * (h00 + h0m);
    const double diag =
        1.0 + (P.gamma - 1.0) * h * h * ((hhp_x + hhm_x) / (P.dx * P.dx) + (hhp_y + hhm_y) / (P.dy * P.dy));
    tdiag[n] = diag * P.dx * P.dy;
  }
};
// momentum correction rho v -= h (g-1) grad E (imex_subsystems.cpp:514-519)
struct k_energy_momentum {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const DevScalars* __restrict__ sc, double* __restrict__ ucon) {
    const long long N = P.N;
    const double h = sc->h;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    int i, j;
    cell_of(P, n, i, j);
    const double* E = ucon + 4 * N;
    ucon[N + n] -= h * (1 / (2 * P.dx)) * (P.gamma - 1) * (E[cid(P, i + 1, j)] - E[cid(P, i - 1, j)]);
    ucon[2 * N + n] -= h * (1 / (2 * P.dy)) * (P.gamma - 1) * (E[cid(P, i, j + 1)] - E[cid(P, i, j - 1)]);
  }
};

// B* right-hand side (imex_subsystems.cpp:549-615) and initial guess x0 = Qe B
struct k_magnetic_rhs_B {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const DevScalars* __restrict__ sc, const double* __restrict__ ucon,
                                   const double* __restrict__ Qe, const double* __restrict__ Qs,
                                   const double* __restrict__ pe, double* __restrict__ b, double* __restrict__ x0) {
    const long long N = P.N;
    const double h = sc->h;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    long long nb[9];
    neighbours(P, n, nb);
    const double* arr[4] = {ucon, Qe, pe, Qs};
    auto ld = [&](int a, int k, long long m) { return __ldg(arr[a] + k * N + m); };
    double out[3];
    mag_rhs_B_cell<double>(P, h, nb, ld, out);
    b[n] = out[0];
    b[N + n] = out[1];
    b[2 * N + n] = out[2];
    x0[n] = Qe[5 * N + n];
    x0[N + n] = Qe[6 * N + n];
    x0[2 * N + n] = Qe[7 * N + n];
  }
};
// ---- local Lax-Friedrichs dissipation (GLF off)
// The speed of cell m along dir (0: x, 1: y) from its conserved state Q:
// 0.5 (|v| + sqrt(v^2 + 4 |B|^2 / rho)) of prim(Q) (implicit_operators.cpp:324-335, 473-480,
// ct_flux.cpp:81-84)
__device__ __forceinline__ double lf_speed(const double* __restrict__ Q, long long N, long long m, int dir) {
  const double rho = __ldg(Q + m), vm = __ldg(Q + (1 + dir) * N + m);
  const double b5 = __ldg(Q + 5 * N + m), b6 = __ldg(Q + 6 * N + m), b7 = __ldg(Q + 7 * N + m);
  const double v = vm / rho;
  return 0.5 * (fabs(v) + sqrt(v * v + 4.0 * (b5 * b5 + b6 * b6 + b7 * b7) / rho));
}
// the pressure viscosity's speed of cell m: |v_dir| (MaterialSpeedp) or |B_dir| / sqrt(rho)
// (AlfvenSpeedp) of prim(Q) (implicit_operators.cpp:587-597)
__device__ __forceinline__ double pv_speed(const DevParams& P, const double* __restrict__ Q, long long N, long long m,
                                           int dir) {
  if (P.add_pvisc == IMEX_MaterialSpeedp) return fabs(__ldg(Q + (1 + dir) * N + m) / __ldg(Q + m));
  return fabs(__ldg(Q + (5 + dir) * N + m) / sqrt(__ldg(Q + m)));
}
// CollectMagFluxes (ct_flux.cpp:5-130) (collect_cell), GLF or local dissipation
struct k_collect_mag_fluxes {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const DevScalars* __restrict__ sc, const double* __restrict__ ucon,
                                       const double* __restrict__ Qe, const double* __restrict__ pe,
                                       double* __restrict__ Fx, double* __restrict__ Fy) {
    const long long N = P.N;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    long long nb[9];
    neighbours(P, n, nb);
    const double* arr[3] = {ucon, Qe, pe};
    auto ld = [&](int a, int k, long long m) { return __ldg(arr[a] + k * N + m); };
    double bmax[2] = {sc->B_max_x, sc->B_max_y};
    if (!P.GLF) {  // the larger speed of the two cells of each face (ct_flux.cpp:79-87, 114-122)
      bmax[0] = fmax(lf_speed(Qe, N, n, 0), lf_speed(Qe, N, nb[NB_E], 0));
      bmax[1] = fmax(lf_speed(Qe, N, n, 1), lf_speed(Qe, N, nb[NB_N], 1));
    }
    double out[2];
    collect_cell<double>(P, sc->h, bmax, nb, ld, out);
    Fx[n] = out[0];
    Fy[n] = out[1];
  }
};

// A** right-hand side (imex_subsystems.cpp:18-51), x0 = A
struct k_magnetic_rhs_A {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const DevScalars* __restrict__ sc, const double* __restrict__ ucon,
                                   const double* __restrict__ Qe, const double* __restrict__ pe,
                                   const double* __restrict__ A_s, double* __restrict__ b, double* __restrict__ irho) {
    const long long N = P.N;
    const double h = sc->h;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    int i, j;
    cell_of(P, n, i, j);
    // every input first, so that the divisions do not serialise the loads; irho (fast
    // arithmetic, else null) receives 1/rho of u_con for the A-form operator
    const double Bxn = Qe[5 * N + n], Byn = Qe[6 * N + n], Bzn = Qe[7 * N + n];
    const double rho = ucon[n], m1 = ucon[N + n], m2 = ucon[2 * N + n], m3 = ucon[3 * N + n];
    const double pxp = pe[cid(P, i + 1, j)], pxm = pe[cid(P, i - 1, j)], pyp = pe[cid(P, i, j + 1)],
                 pym = pe[cid(P, i, j - 1)];
    const double a0 = A_s[n], a1 = A_s[N + n], a2 = A_s[2 * N + n];
    const double Sx = m1 / rho - h / rho * (pxp - pxm) / (2.0 * P.dx);
    const double Sy = m2 / rho - h / rho * (pyp - pym) / (2.0 * P.dy);
    const double Sz = m3 / rho;
    b[n] = a0 - h * (Byn * Sz - Bzn * Sy);
    b[N + n] = a1 - h * (Bzn * Sx - Bxn * Sz);
    b[2 * N + n] = a2 - h * (Bxn * Sy - Byn * Sx);
    if (irho) irho[n] = 1.0 / rho;
  }
};
// global A-viscosity maxima of prim(Qs) over real cells (implicit_operators.cpp:364-374)
struct k_gmax {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, const double* __restrict__ Qs, double* __restrict__ partial) {
    double m0 = 0.0, m1 = 0.0;
    // four cells per round, all loaded before the first division (the maxima do not depend
    // on the order cells are visited in)
    constexpr int kU = 4;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long n0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; n0 < P.N; n0 += kU * stride) {
      double c[kU][8];
  #pragma unroll
      for (int u = 0; u < kU; ++u)
        if (n0 + u * stride < P.N) load_cell<8>(Qs, P.N, n0 + u * stride, c[u]);
  #pragma unroll
      for (int u = 0; u < kU; ++u) {
        if (n0 + u * stride >= P.N) break;
        double p[8];
        con2pri(P, p, c[u]);
        double Bsq = p[5] * p[5] + p[6] * p[6] + p[7] * p[7];
        m0 = fmax(m0, 0.5 * (fabs(p[1]) + sqrt(p[1] * p[1] + 4.0 * Bsq / p[0])));
        m1 = fmax(m1, 0.5 * (fabs(p[2]) + sqrt(p[2] * p[2] + 4.0 * Bsq / p[0])));
      }
    }
    __shared__ double sh[2][kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
      m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
      m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
    }
    if ((threadIdx.x & 31) == 0) {
      sh[0][threadIdx.x >> 5] = m0;
      sh[1][threadIdx.x >> 5] = m1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0, b = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        a = fmax(a, sh[0][w]);
        b = fmax(b, sh[1][w]);
      }
      partial[2 * blockIdx.x] = a;
      partial[2 * blockIdx.x + 1] = b;
    }
  }
};
// r = 1 / a over n values (the A-form operator's 1/rho in the fast arithmetic)
struct k_recip {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, const double* __restrict__ a, double* __restrict__ r, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) r[i] = 1.0 / a[i];
  }
};
constexpr int kGmaxThreads = 1024;  // one block reduces the per-CTA maxima of a whole plane
struct k_gmax_finalize {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, const double* __restrict__ partial, int nblk, DevScalars* sc) {
    double a = 0.0, b = 0.0;
    for (int k = threadIdx.x; k < nblk; k += blockDim.x) {
      a = fmax(a, partial[2 * k]);
      b = fmax(b, partial[2 * k + 1]);
    }
    __shared__ double sh[2][32];  // one slot per warp of up to 1024 threads
    for (int o = 16; o > 0; o >>= 1) {
      a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
      b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    if ((threadIdx.x & 31) == 0) {
      sh[0][threadIdx.x >> 5] = a;
      sh[1][threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
        a = fmax(a, sh[0][w]);
        b = fmax(b, sh[1][w]);
      }
      sc->gmax_bx = a;
      sc->gmax_by = b;
    }
  }
};
// ---- face viscosities of the local dissipation
enum { LV_MAG_B = 0, LV_MAG_A = 1, LV_PRES = 2 };
// The face viscosities of one solve, frozen like its other coefficients: plane f of lv holds,
// for every cell, the face x+ (f = 0), x- (1), y+ (2) or y- (3), as the operator multiplies it.
//   LV_MAG_B: max(b_c, b_nb) d from prim(Qe)        (implicit_operators.cpp:323-345)
//   LV_MAG_A: (b_c + b_nb) / 2 d from prim(Qs)      (implicit_operators.cpp:472-486)
//   LV_PRES:  (eta_nb + eta_c) / 2 max(s_c, s_nb) d (implicit_operators.cpp:584-607)
// d is dx for the x faces and dy for the y faces; a neighbour outside a transmissive
// direction is the nearest interior cell.
struct k_local_visc {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams P, int mode, const double* __restrict__ Q, const double* __restrict__ eta,
                               double* __restrict__ lv) {
    const long long N = P.N;
    const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    int i, j;
    cell_of(P, n, i, j);
    const long long nbr[4] = {cid(P, i + 1, j), cid(P, i - 1, j), cid(P, i, j + 1), cid(P, i, j - 1)};
    double own[2], out[4];
    if (mode == LV_PRES) {
      own[0] = pv_speed(P, Q, N, n, 0);
      own[1] = pv_speed(P, Q, N, n, 1);
      const double ec = __ldg(eta + n);
  #pragma unroll
      for (int f = 0; f < 4; ++f) {
        const int dir = f >> 1;
        const double nu = fmax(own[dir], pv_speed(P, Q, N, nbr[f], dir)) * (dir ? P.dy : P.dx);
        out[f] = 0.5 * (__ldg(eta + nbr[f]) + ec) * nu;
      }
    } else {
      own[0] = lf_speed(Q, N, n, 0);
      own[1] = lf_speed(Q, N, n, 1);
  #pragma unroll
      for (int f = 0; f < 4; ++f) {
        const int dir = f >> 1;
        const double b = lf_speed(Q, N, nbr[f], dir), d = dir ? P.dy : P.dx;
        out[f] = mode == LV_MAG_B ? fmax(own[dir], b) * d : 0.5 * (own[dir] + b) * d;
      }
    }
  #pragma unroll
    for (int f = 0; f < 4; ++f) lv[f * N + n] = out[f];
  }
};
// B = curl A after the A solve (imex_subsystems.cpp:65-72)
template <bool kOpen>
struct k_curl_A {
  IMEX_BOUNDS(0, 0)
  static __device__ __forceinline__ void run(IMEX_BLK, DevParams Pin, const double* __restrict__ A, double* __restrict__ ucon) {
    const DevParams P = bc_params<kOpen>(Pin);
    const long long N = P.N;
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= N) return;
    int i, j;
    cell_of(P, n, i, j);
    auto Ak = [&](int k, int di, int dj) { return a_ghost(P, A + k * N, i + di, j + dj); };
    ucon[5 * N + n] = 1 / (2.0 * P.dy) * (Ak(2, 0, 1) - Ak(2, 0, -1));
    ucon[6 * N + n] = -1 / (2.0 * P.dx) * (Ak(2, 1, 0) - Ak(2, -1, 0));
    ucon[7 * N + n] = 1 / (2.0 * P.dx) * (Ak(1, 1, 0) - Ak(1, -1, 0)) - 1 / (2.0 * P.dy) * (Ak(0, 0, 1) - Ak(0, 0, -1));
  }
};

// ------------------------------------------------------------------ plain operator application
template <class Op>
__global__ void __launch_bounds__(NT) k_apply(Op op, Tiling T, const double* x, double* Ax) {
  op.bind();
  extern __shared__ __align__(16) unsigned char dsm[];
  TileBuf<Op>& tb = *reinterpret_cast<TileBuf<Op>*>(dsm);
  for (int t = blockIdx.x; t < T.ntiles; t += gridDim.x) {
    const int x0 = (t % T.tiles_x) * TXo<Op>, y0 = (t / T.tiles_x) * TYo<Op>;
    fill_tile(op, tb, T, x0, y0, [&](const long long* c, double (*v)[Op::M]) {
#pragma unroll
      for (int r = 0; r < FillQ<Op>; ++r)
#pragma unroll
        for (int m = 0; m < Op::M; ++m) v[r][m] = x[m * T.N + c[r]];
    });
#pragma unroll
    for (int r = 0; r < CPTo<Op>; ++r) {
      const Cell k = tile_cell<Op>(T, x0, y0, r);
      if (!k.in) continue;
      double ax[Op::M];
      op.matvec(tb, k.lx, k.ly, k.c, ax);
#pragma unroll
      for (int m = 0; m < Op::M; ++m) Ax[m * T.N + k.c] = ax[m];
    }
    __syncthreads();
  }
}

// Device-wide barrier self-test: `iters` barriers over the launched CTAs plus
// `phantom` CTAs that are never launched (so with phantom > 0 the bounded wait
// must run out and report IMEX_ERR_SYNC).  Block 0 reports clock cycles.
__global__ void k_barrier_selftest(SyncState* sync, unsigned phantom, int iters, DevStats* st,
                                   long long* cycles) {
  const unsigned nblk = gridDim.x + phantom;
  long long t0 = clock64();
  for (int k = 0; k < iters; ++k) {
    if (!grid_barrier(sync, nblk)) {
      if (threadIdx.x == 0) atomicMax(&st->status, (int)IMEX_ERR_SYNC);
      return;
    }
  }
  if (threadIdx.x == 0 && blockIdx.x == 0) *cycles = clock64() - t0;
}

}  // namespace

// ================================================================== host side
#define LAUNCH_CHECK(ctx, what)                              \
  do {                                                       \
    cudaError_t e_ = cudaGetLastError();                     \
    if (e_ != cudaSuccess) return cuda_check(ctx, e_, what); \
  } while (0)
#define BYTES(vals) ((double)(vals) * 8.0 * (double)ctx->N)

namespace {

// CTAs of a cooperative launch of `kernel` with `smem` bytes of dynamic shared memory
int coop_blocks_smem(imex_ctx* ctx, const void* kernel, const Tiling& T, size_t smem) {
  int per_sm = 0;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, NT, smem);
  if (per_sm < 1) per_sm = 1;
  if (per_sm > 4) per_sm = 4;
  int nb = per_sm * ctx->num_sms;
  if (nb > T.ntiles) nb = T.ntiles;
  if (nb > ctx->max_blocks) nb = ctx->max_blocks;
  if (nb < 1) nb = 1;
  return nb;
}
template <class Op>
int coop_blocks(imex_ctx* ctx, const void* kernel, const Tiling& T) {
  return coop_blocks_smem(ctx, kernel, T, sizeof(SolveSmem<Op>));
}

GmresWork make_work(imex_ctx* ctx, const Tiling& T, int nblk, int fam) {
  GmresWork g{};
  g.fam = fam;
  g.V = ctx->V;
  g.AV = ctx->AV;
  g.partial = ctx->partial;
  g.sync = ctx->sync;
  g.st = ctx->st;
  g.kmax = ctx->cfg.gmres_restart;
  // 0 = the system's dimension, as the reference's outmax = dim (implicit_operators.cpp:802):
  // 3N for the magnetic systems and the adjoint's, N for the pressure and energy systems
  const long long width = (fam == F_GMRES_MAG_B || fam == F_GMRES_MAG_A || fam == F_ADJOINT) ? 3 : 1;
  const long long dim = width * T.N;
  g.max_restarts = ctx->cfg.gmres_max_restarts > 0 ? ctx->cfg.gmres_max_restarts
                                                   : (int)(dim > 2000000000LL ? 2000000000LL : dim);
  g.nblk = nblk;
  g.tol = ctx->P.GMREStol;
  g.tol_abs = ctx->P.GMREStol;
  g.T = T;
  return g;
}
// FP32 Krylov workspace of the mixed form; inner solves stop at a relative residual of
// mixed_inner_tol (plus `tol_abs`), after at most `max_restarts` cycles
GmresWorkT<float> make_work_mixed(imex_ctx* ctx, const Tiling& T, int nblk, int fam, int max_restarts,
                                  double tol_abs) {
  const GmresWork d = make_work(ctx, T, nblk, fam);
  GmresWorkT<float> g{};
  g.V = ctx->Vf;
  g.AV = ctx->AVf;
  g.partial = d.partial;
  g.sync = d.sync;
  g.st = d.st;
  g.kmax = d.kmax;
  g.max_restarts = max_restarts;
  g.nblk = nblk;
  g.fam = fam;
  g.tol = ctx->cfg.mixed_inner_tol;
  g.tol_abs = tol_abs;
  g.T = T;
  return g;
}
// whether solves of the given kind (IMEX_MIXED_*) take the mixed form
bool mixed(const imex_ctx* ctx, int kind) {
  return ctx->cfg.precision == IMEX_PRECISION_MIXED && (ctx->cfg.mixed_solves & kind) != 0;
}
// tolerance of the FP64 refinement of a mixed solve: mixed_outer_tol, or GMREStol when that is 0
double mixed_outer_tol(const imex_ctx* ctx) {
  return ctx->cfg.mixed_outer_tol > 0.0 ? ctx->cfg.mixed_outer_tol : ctx->P.GMREStol;
}

}  // namespace
__global__ void k_reset_sync(SyncState* s, long long limit) {
  s->count = 0;
  s->abort = 0;
  s->wait_cycles = limit;
}
namespace {
// every device-wide wait gives up after ~barrier_timeout_s (a wait never legitimately lasts that
// long); counted in SM cycles at the maximum clock, so a slower clock only lengthens the bound.
// The clock rate is read once at creation: querying it per launch stalls the host.
long long wait_cycles(const imex_ctx* ctx) {
  const double khz = ctx->clock_khz > 0 ? (double)ctx->clock_khz : 2.0e6;
  return (long long)(ctx->barrier_timeout_s * khz * 1e3) + 1;
}
imex_status reset_sync(imex_ctx* ctx) {
  k_reset_sync<<<1, 1, 0, ctx->stream>>>(ctx->sync, wait_cycles(ctx));
  return cuda_check(ctx, cudaGetLastError(), "sync reset");
}

template <class K, class... Args>
imex_status launch_coop_smem(imex_ctx* ctx, K kernel, int nblk, size_t smem, Args... args) {
  imex_status s = reset_sync(ctx);
  if (s != IMEX_OK) return s;
  void* params[] = {(void*)&args...};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)kernel, dim3(nblk), dim3(NT), params, smem, ctx->stream);
  return cuda_check(ctx, e, "cooperative launch");
}
template <class Op, class K, class... Args>
imex_status launch_coop(imex_ctx* ctx, K kernel, int nblk, Args... args) {
  return launch_coop_smem(ctx, kernel, nblk, sizeof(SolveSmem<Op>), args...);
}

PressureOp make_pressure_op(imex_ctx* ctx) {
  PressureOp op{};
  op.P = ctx->P;
  op.sc = ctx->sc;
  op.hh = ctx->hh;
  op.eta = ctx->eta;
  op.rho = ctx->cons;
  op.vscale = ctx->vscale;
  op.tdiag = ctx->tdiag;
  op.vdiag = ctx->vdiag;
  op.lv = ctx->P.add_pvisc == IMEX_Noaddvisp ? nullptr : ctx->lvp;
  op.jac = 0;
  return op;
}
EnergyOp make_energy_op(imex_ctx* ctx) {
  EnergyOp op{};
  op.P = ctx->P;
  op.sc = ctx->sc;
  op.hh = ctx->hh;
  op.tdiag = ctx->tdiag;
  return op;
}
MagneticBOp make_magB_op(imex_ctx* ctx) {
  MagneticBOp op{};
  op.P = ctx->P;
  op.sc = ctx->sc;
  op.Qe = ctx->Qe;
  op.rho = ctx->cons;
  op.lv = ctx->lvm;
  return op;
}
template <int kTX = TX, int kTY = TY>
MagneticBFastOpT<double, kTX, kTY> make_magB_fast_op(imex_ctx* ctx) {
  MagneticBFastOpT<double, kTX, kTY> op{};
  static_cast<MagneticBCoef&>(op) = static_cast<const MagneticBCoef&>(make_magB_op(ctx));
  return op;
}
template <bool kOpen = false>
MagneticAOpT<double, kOpen> make_magA_op(imex_ctx* ctx) {
  MagneticAOpT<double, kOpen> op{};
  op.P = ctx->P;
  op.sc = ctx->sc;
  op.Qe = ctx->Qe;
  op.rho = ctx->cons;
  op.irho = ctx->P.fast ? ctx->irho : nullptr;
  op.lv = ctx->lvm;
  op.add_bvisc = ctx->P.add_bvisc;
  return op;
}

template <class Op>
void launch_apply(imex_ctx* ctx, const Op& o, int nb, const Tiling& T, const double* x, double* Ax) {
  const size_t smem = sizeof(TileBuf<Op>);
  cudaFuncSetAttribute((const void*)k_apply<Op>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  prof_begin(ctx);
  k_apply<Op><<<nb, NT, smem, ctx->stream>>>(o, T, x, Ax);
  prof_end(ctx, F_APPLY, (double)(2 * Op::M + Op::COEF) * 8.0 * (double)T.N, 1);
}

// hh and the right-hand side / Jacobi scale of the energy solve
imex_status energy_setup(imex_ctx* ctx) {
  const DevParams& P = ctx->P;
  int nb = blocks_for(P.N);
  prof_begin(ctx);
  launch<k_energy_coeffs>(ctx, nb, kThreads, 0, ctx->stream, P, ctx->Qe, ctx->cons, ctx->hh);
  LAUNCH_CHECK(ctx, "k_energy_coeffs");
  prof_end(ctx, F_PRES_SETUP, BYTES(10), 1);
  prof_begin(ctx);
  launch<k_energy_rhs>(ctx, nb, kThreads, 0, ctx->stream, P, ctx->sc, ctx->cons, ctx->hh, ctx->pb, ctx->tdiag);
  LAUNCH_CHECK(ctx, "k_energy_rhs");
  prof_end(ctx, F_PRES_RHS, BYTES(6), 1);
  return IMEX_OK;
}
imex_status energy_momentum(imex_ctx* ctx) {
  int nb = blocks_for(ctx->P.N);
  prof_begin(ctx);
  launch<k_energy_momentum>(ctx, nb, kThreads, 0, ctx->stream, ctx->P, ctx->sc, ctx->cons);
  LAUNCH_CHECK(ctx, "k_energy_momentum");
  prof_end(ctx, F_MOMENTUM, BYTES(5), 1);
  return IMEX_OK;
}
// the face viscosities of the local dissipation (GLF off) for the magnetic solve (from Qe,
// or Qs in the A form) or the pressure solve (from Qe and eta); nothing with GLF
imex_status local_visc(imex_ctx* ctx, int mode) {
  const DevParams& P = ctx->P;
  if (P.GLF || (mode == LV_PRES && P.add_pvisc == IMEX_Noaddvisp)) return IMEX_OK;
  const int nb = blocks_for(P.N);
  prof_begin(ctx);
  if (mode == LV_PRES)
    launch<k_local_visc>(ctx, nb, kThreads, 0, ctx->stream, P, mode, ctx->Qe, ctx->eta, ctx->lvp);
  else
    launch<k_local_visc>(ctx, nb, kThreads, 0, ctx->stream, P, mode, mode == LV_MAG_A ? ctx->Qs : ctx->Qe, nullptr, ctx->lvm);
  LAUNCH_CHECK(ctx, "k_local_visc");
  prof_end(ctx, mode == LV_PRES ? F_PRES_SETUP : F_MAG_RHS, BYTES(mode == LV_PRES ? 8 : 10), 1);
  return IMEX_OK;
}
int mag_visc_mode(const imex_ctx* ctx) { return ctx->P.magfield == IMEX_PotentialA ? LV_MAG_A : LV_MAG_B; }

imex_status pressure_setup(imex_ctx* ctx) {
  const DevParams& P = ctx->P;
  int nb = blocks_for(P.N);
  prof_begin(ctx);
  IMEX_LAUNCH_BC(P, k_pressure_coeffs, nb, kThreads, 0, ctx->stream, P, ctx->Qe, ctx->cons, ctx->hQe, ctx->pe, ctx->hh,
                 ctx->vscale, ctx->rv, &ctx->sc->bkey[0][0]);
  LAUNCH_CHECK(ctx, "k_pressure_coeffs");
  IMEX_LAUNCH_BC(P, k_pressure_tdiag, nb, kThreads, 0, ctx->stream, P, ctx->sc, ctx->hh, ctx->tdiag);
  LAUNCH_CHECK(ctx, "k_pressure_tdiag");
  prof_end(ctx, F_PRES_SETUP, BYTES(12 + 2), 2);
  imex_status s = launch_shock(ctx, ctx->Qe, ctx->eta);
  if (s != IMEX_OK) return s;
  return local_visc(ctx, LV_PRES);
}

// One GMRES solve with operator o: the plain FP64 kernel, or in the mixed form the FP64
// refinement kernel around FP32 inner cycles.
template <class Op>
imex_status gmres_run(imex_ctx* ctx, const Op& o, int fam, double* x, const double* b, int kind) {
  const Tiling T = make_tiling_for<Op>(ctx);
  if (!mixed(ctx, kind)) {
    auto kern = k_gmres<Op>;
    const int nb = coop_blocks<Op>(ctx, (const void*)kern, T);
    GmresWork g = make_work(ctx, T, nb, fam);
    prof_begin(ctx);
    imex_status s = launch_coop<Op>(ctx, kern, nb, o, g, x, b);
    prof_end(ctx, fam, 0.0, 1);
    return s;
  }
  auto kern = k_gmres_mixed<Op>;
  const size_t smem = sizeof(MixedSmem<Op>);
  const int nb = coop_blocks_smem(ctx, (const void*)kern, T, smem);
  GmresWorkT<float> g = make_work_mixed(ctx, T, nb, fam, 1, 0.0);
  prof_begin(ctx);
  imex_status s = launch_coop_smem(ctx, kern, nb, smem, o, g, x, ctx->mcor, ctx->mres, b, ctx->cfg.mixed_max_refine,
                                   mixed_outer_tol(ctx));
  prof_end(ctx, fam, 0.0, 1);
  return s;
}

imex_status gmres_launch(imex_ctx* ctx, int op, double* x, const double* b) {
  if (op == IMEX_OP_PRESSURE_L || op == IMEX_OP_PRESSURE_J) {
    PressureOp o = make_pressure_op(ctx);
    o.jac = op == IMEX_OP_PRESSURE_J;
    return gmres_run(ctx, o, F_GMRES_PRES, x, b, IMEX_MIXED_PRESSURE);
  } else if (op == IMEX_OP_MAGNETIC_B) {
    if (ctx->P.fast)
      return gmres_run(ctx, make_magB_fast_op<>(ctx), F_GMRES_MAG_B, x, b, IMEX_MIXED_MAGNETIC | IMEX_MIXED_MAGNETIC_B);
    return gmres_run(ctx, make_magB_op(ctx), F_GMRES_MAG_B, x, b, IMEX_MIXED_MAGNETIC | IMEX_MIXED_MAGNETIC_B);
  } else if (op == IMEX_OP_MAGNETIC_A) {
    if (ctx->P.xclamp || ctx->P.yclamp)
      return gmres_run(ctx, make_magA_op<true>(ctx), F_GMRES_MAG_A, x, b, IMEX_MIXED_MAGNETIC);
    return gmres_run(ctx, make_magA_op(ctx), F_GMRES_MAG_A, x, b, IMEX_MIXED_MAGNETIC);
  } else if (op == IMEX_OP_ENERGY) {
    return gmres_run(ctx, make_energy_op(ctx), F_GMRES_ENERGY, x, b, IMEX_MIXED_PRESSURE);
  }
  return set_error(ctx, IMEX_ERR_UNSUPPORTED, "operator not available");
}

bool on_device(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// The same GMRES launch as gmres_launch, with every work array carved out of the
// caller's fixed scratch [base, base + capacity) instead of the context's buffers:
//   barrier state | partial sums (2 x CTAs x NP) | V ((restart+1) vectors) | AV (2) | x, b staging (host only)
// Nothing here allocates; a solve that does not fit is rejected before any work.
template <class Op>
imex_status gmres_noalloc_op(imex_ctx* ctx, const Op& o, int fam, double* x, const double* b, unsigned char* base,
                             size_t capacity) {
  const Tiling T = make_tiling_for<Op>(ctx);
  auto kern = k_gmres<Op>;
  const int nb = coop_blocks<Op>(ctx, (const void*)kern, T);
  const size_t n = (size_t)Op::M * (size_t)T.N;
  const bool hx = !on_device(x), hb = !on_device(b);
  size_t used = 0;
  auto take = [&](size_t bytes) {
    const size_t at = used;
    used += (bytes + 255) & ~(size_t)255;
    return at;
  };
  const size_t o_sync = take(sizeof(SyncState));
  const size_t o_part = take((size_t)2 * nb * NP * sizeof(double));
  const size_t o_V = take(((size_t)ctx->cfg.gmres_restart + 1) * n * sizeof(double));
  const size_t o_AV = take(2 * n * sizeof(double));
  const size_t o_x = hx ? take(n * sizeof(double)) : 0;
  const size_t o_b = hb ? take(n * sizeof(double)) : 0;
  if (used > capacity) {
    char msg[256];
    snprintf(msg, sizeof(msg),
             "imex_gmres_noalloc: this solve needs %zu bytes of scratch (restart %d, %zu unknowns), "
             "the static scratch holds %zu",
             used, ctx->cfg.gmres_restart, n, capacity);
    return set_error(ctx, IMEX_ERR_INVALID, msg);
  }
  GmresWork g = make_work(ctx, T, nb, fam);
  g.sync = reinterpret_cast<SyncState*>(base + o_sync);
  g.partial = reinterpret_cast<double*>(base + o_part);
  g.V = reinterpret_cast<double*>(base + o_V);
  g.AV = reinterpret_cast<double*>(base + o_AV);
  double* xd = hx ? reinterpret_cast<double*>(base + o_x) : x;
  const double* bd = hb ? reinterpret_cast<const double*>(base + o_b) : b;
  cudaError_t e = cudaSuccess;
  if (hx) e = cudaMemcpyAsync(xd, x, n * sizeof(double), cudaMemcpyDefault, ctx->stream);
  if (hb && e == cudaSuccess) e = cudaMemcpyAsync((void*)bd, b, n * sizeof(double), cudaMemcpyDefault, ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "imex_gmres_noalloc: vector upload");
  // the barrier state must start at zero on every call
  k_reset_sync<<<1, 1, 0, ctx->stream>>>(g.sync, wait_cycles(ctx));
  LAUNCH_CHECK(ctx, "imex_gmres_noalloc: sync reset");
  void* params[] = {(void*)&o, (void*)&g, (void*)&xd, (void*)&bd};
  e = cudaLaunchCooperativeKernel((const void*)kern, dim3(nb), dim3(NT), params, sizeof(SolveSmem<Op>), ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "imex_gmres_noalloc: cooperative launch");
  ctx->kernel_launches += 2;
  if (hx) e = cudaMemcpyAsync(x, xd, n * sizeof(double), cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_check(ctx, e, "imex_gmres_noalloc: solve");
}

// keys: b is this context's pb just written by k_pressure_rhs into key slot `keys` - 1 (the
// floor slope's inputs min b, max V); 0: the solve reduces them itself
imex_status newton_launch(imex_ctx* ctx, double* p, const double* b, int keys = 0) {
  const DevParams& P = ctx->P;
  PressureOp o = make_pressure_op(ctx);
  if (!P.floor_on && P.eos_type == IMEX_IDEAL_GAS)  // a single linear GMRES with L (implicit_operators.cpp:664-668)
    return gmres_run(ctx, o, F_NEWTON, p, b, IMEX_MIXED_PRESSURE);
  const Tiling T = make_tiling(ctx->nx, ctx->ny, ctx->P.xclamp, ctx->P.yclamp);
  NewtonArgs na{};
  na.p = p;
  na.pf = ctx->pf;
  na.g = ctx->pg;
  na.dp = ctx->pdp;
  na.vdiag = ctx->vdiag;
  na.b = b;
  na.sc = ctx->sc;
  na.bkeys = keys ? ctx->sc->bkey[keys - 1] : nullptr;
  imex_status s;
  // Above 2^21 cells (between 1024^2 and 2048^2) the solve's planes outgrow the 126 MB L2 and
  // the 3-CTA instance is faster (2048^2 vortex sheet: 5.71 -> 4.96 ms of Newton per step;
  // 1024^2: 1.68 -> 1.74, so that size keeps the 2-CTA instance).
  const bool wide = ctx->N >= (size_t(1) << 21);
  prof_begin(ctx);
  if (!mixed(ctx, IMEX_MIXED_PRESSURE)) {
    auto kern = P.eos_type == IMEX_IDEAL_GAS ? (wide ? k_nested_newton<double, false, 3> : k_nested_newton<double, false>)
                                             : (wide ? k_nested_newton<double, true, 3> : k_nested_newton<double, true>);
    const size_t smem = sizeof(NewtonSmem<double>);
    const int nb = coop_blocks_smem(ctx, (const void*)kern, T, smem);
    GmresWork g = make_work(ctx, T, nb, F_NEWTON);
    s = launch_coop_smem(ctx, kern, nb, smem, o, g, na);
  } else {
    auto kern = P.eos_type == IMEX_IDEAL_GAS ? (wide ? k_nested_newton<float, false, 3> : k_nested_newton<float, false>)
                                             : (wide ? k_nested_newton<float, true, 3> : k_nested_newton<float, true>);
    const size_t smem = sizeof(NewtonSmem<float>);
    const int nb = coop_blocks_smem(ctx, (const void*)kern, T, smem);
    GmresWorkT<float> g = make_work_mixed(ctx, T, nb, F_NEWTON, make_work(ctx, T, nb, F_NEWTON).max_restarts,
                                          ctx->P.GMREStol);
    s = launch_coop_smem(ctx, kern, nb, smem, o, g, na);
  }
  prof_end(ctx, F_NEWTON, 0.0, 1);
  return s;
}

// ---- batched solves (host side)
// The members are spread over one or more cooperative launches (chunks) of the kernel's
// co-resident capacity C (its occupancy, capped at 4 CTAs per SM, times the SMs).  Members
// are sorted by work (tiles) and dealt to L chunks in snake order, with L large enough that
// no chunk holds more than C/2 members, so every chunk carries about the same work and has
// room to give large members many CTAs.  Within a chunk every member gets at least one CTA
// and at most one per tile, the rest in proportion to its tiles.
template <class ShapeOp, class Job, class K, class Make>
imex_status add_chunks(BatchSolvePlan* plan, const std::vector<imex_ctx*>& members, K kernel, size_t smem,
                       Make make_job) {
  imex_ctx* c0 = members[0];
  cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)kernel, NT, smem);
  if (per_sm > 4) per_sm = 4;
  if (per_sm < 1) return set_error(c0, IMEX_ERR_CUDA, "batched solve kernel does not fit on an SM");
  const int cap = per_sm * c0->num_sms;
  const long long limit = wait_cycles(c0);
  const int nm = (int)members.size();
  auto tiles = [&](int m) { return make_tiling(members[m]->nx, members[m]->ny, 0, 0, TXo<ShapeOp>, TYo<ShapeOp>).ntiles; };
  std::vector<int> order(nm);
  for (int m = 0; m < nm; ++m) order[m] = m;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return tiles(a) > tiles(b); });
  const int per_chunk = cap / 2 > 0 ? cap / 2 : 1;
  const int L = (nm + per_chunk - 1) / per_chunk;
  std::vector<std::vector<int>> groups(L);
  for (int i = 0; i < nm; ++i) {
    const int r = i % (2 * L);
    groups[r < L ? r : 2 * L - 1 - r].push_back(order[i]);
  }
  for (const std::vector<int>& grp : groups) {
    if (grp.empty()) continue;
    const int n = (int)grp.size();
    double tiles_sum = 0.0;
    for (int m : grp) tiles_sum += tiles(m);
    std::vector<int> alloc(n, 1);
    const int left = cap - n;
    for (int k = 0; k < n; ++k) {
      const int nt = tiles(grp[k]);
      int extra = (int)((double)left * nt / tiles_sum);
      if (extra > nt - 1) extra = nt - 1;
      alloc[k] += extra;
    }
    std::vector<Job> jobs;
    std::vector<int> map;
    std::vector<SyncState*> syncs;
    int first = 0;
    for (int k = 0; k < n; ++k) {
      imex_ctx* m = members[grp[k]];
      jobs.push_back(make_job(m, make_tiling_for<ShapeOp>(m), first, alloc[k]));
      for (int q = 0; q < alloc[k]; ++q) map.push_back(k);
      syncs.push_back(m->sync);
      first += alloc[k];
    }
    Job* d_jobs = nullptr;
    int* d_map = nullptr;
    SyncState** d_syncs = nullptr;
    cudaError_t e = cudaMalloc(&d_jobs, jobs.size() * sizeof(Job));
    if (e == cudaSuccess) e = cudaMalloc(&d_map, map.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&d_syncs, syncs.size() * sizeof(SyncState*));
    if (d_jobs) plan->dev.push_back(d_jobs);
    if (d_map) plan->dev.push_back(d_map);
    if (d_syncs) plan->dev.push_back(d_syncs);
    if (e == cudaSuccess) e = cudaMemcpy(d_jobs, jobs.data(), jobs.size() * sizeof(Job), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_map, map.data(), map.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(d_syncs, syncs.data(), syncs.size() * sizeof(SyncState*), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_check(c0, e, "batched solve set-up");
    const int nctas = first;
    BatchChunk ch;
    ch.ctas = nctas;
    ch.members = n;
    ch.launch = [=](cudaStream_t st) {
      k_reset_syncs<<<(n + 255) / 256, 256, 0, st>>>(d_syncs, n, limit);
      cudaError_t e2 = cudaGetLastError();
      if (e2 != cudaSuccess) return e2;
      const Job* dj = d_jobs;
      const int* dm = d_map;
      void* params[] = {(void*)&dj, (void*)&dm};
      return cudaLaunchCooperativeKernel((const void*)kernel, dim3(nctas), dim3(NT), params, smem, st);
    };
    plan->chunks.push_back(ch);
  }
  return IMEX_OK;
}

template <class Op>
GmresWork job_work(imex_ctx* m, const Tiling& T, int first, int nblk, int fam) {
  GmresWork g = make_work(m, T, nblk, fam);
  g.first = first;
  return g;
}
GmresWorkT<float> job_work_mixed(imex_ctx* m, const Tiling& T, int first, int nblk, int fam, int max_restarts,
                                 double tol_abs) {
  GmresWorkT<float> g = make_work_mixed(m, T, nblk, fam, max_restarts, tol_abs);
  g.first = first;
  return g;
}

// one GMRES per member with operator make_op(member), plain or mixed
template <class Op, class MakeOp, class Sys>
imex_status add_gmres_chunks(BatchSolvePlan* plan, const std::vector<imex_ctx*>& members, int kind, int fam,
                             MakeOp make_op, Sys system) {
  if (!mixed(members[0], kind)) {
    return add_chunks<Op, GmresJob<Op>>(plan, members, k_gmres_jobs<Op>, sizeof(SolveSmem<Op>),
                                    [&](imex_ctx* m, const Tiling& T, int first, int nblk) {
                                      GmresJob<Op> j{};
                                      j.op = make_op(m);
                                      j.g = job_work<Op>(m, T, first, nblk, fam);
                                      system(m, &j.x, &j.b);
                                      return j;
                                    });
  }
  return add_chunks<Op, MixedJob<Op>>(plan, members, k_gmres_mixed_jobs<Op>, sizeof(MixedSmem<Op>),
                                  [&](imex_ctx* m, const Tiling& T, int first, int nblk) {
                                    MixedJob<Op> j{};
                                    j.op = make_op(m);
                                    j.g = job_work_mixed(m, T, first, nblk, fam, 1, 0.0);
                                    system(m, &j.x, &j.b);
                                    j.xalt = m->mcor;
                                    j.sres = m->mres;
                                    j.max_sweeps = m->cfg.mixed_max_refine;
                                    j.tol = mixed_outer_tol(m);
                                    return j;
                                  });
}

template <class TS>
imex_status add_newton_chunks(BatchSolvePlan* plan, const std::vector<imex_ctx*>& members) {
  // members share the configuration, so one instance serves all of them
  auto kern = members[0]->P.eos_type == IMEX_IDEAL_GAS ? k_nested_newton_jobs<TS, false> : k_nested_newton_jobs<TS, true>;
  return add_chunks<PressureOp, NewtonJob<TS>>(
      plan, members, kern, sizeof(NewtonSmem<TS>),
      [&](imex_ctx* m, const Tiling& T, int first, int nblk) {
        NewtonJob<TS> j{};
        j.op = make_pressure_op(m);
        if constexpr (std::is_same<TS, double>::value) {
          j.gw = job_work<PressureOp>(m, T, first, nblk, F_NEWTON);
        } else {
          j.gw = job_work_mixed(m, T, first, nblk, F_NEWTON, make_work(m, T, nblk, F_NEWTON).max_restarts,
                                m->P.GMREStol);
        }
        j.na.p = m->pp;
        j.na.pf = m->pf;
        j.na.g = m->pg;
        j.na.dp = m->pdp;
        j.na.vdiag = m->vdiag;
        j.na.b = m->pb;
        j.na.sc = m->sc;
        j.na.bkeys = nullptr;  // one plan serves both pressure solves of a stage: reduce in the kernel
        return j;
      });
}

}  // namespace

// The batched solve of one kind for every member (all members share the configuration
// flags that select the solve; each has its own grid, data and restart length).
imex_status batch_solve_build(const std::vector<imex_ctx*>& members, int kind, BatchSolvePlan** out, int tile) {
  if (members.empty()) return IMEX_ERR_INVALID;
  BatchSolvePlan* plan = new BatchSolvePlan();
  imex_ctx* c0 = members[0];
  const DevParams& P = c0->P;
  imex_status s;
  if (kind == BATCH_MAGNETIC) {
    auto sys = [](imex_ctx* m, double** x, const double** b) {
      int op;
      mag_system(m, &op, x, b);
    };
    if (P.magfield == IMEX_PotentialA && (P.xclamp || P.yclamp))  // members share the configuration
      s = add_gmres_chunks<MagneticAOpOpen>(plan, members, IMEX_MIXED_MAGNETIC, F_GMRES_MAG_A, make_magA_op<true>,
                                            sys);
    else if (P.magfield == IMEX_PotentialA)
      s = add_gmres_chunks<MagneticAOp>(plan, members, IMEX_MIXED_MAGNETIC, F_GMRES_MAG_A, make_magA_op<false>, sys);
    else if (P.fast) {  // the tile shape an ensemble chose (imex_batch_set_solve_tile)
      constexpr int mk = IMEX_MIXED_MAGNETIC | IMEX_MIXED_MAGNETIC_B;
      if (tile == 1)
        s = add_gmres_chunks<MagneticBFastOpT<double, 64, 8>>(plan, members, mk, F_GMRES_MAG_B,
                                                              make_magB_fast_op<64, 8>, sys);
      else if (tile == 2)
        s = add_gmres_chunks<MagneticBFastOpT<double, 32, 8>>(plan, members, mk, F_GMRES_MAG_B,
                                                              make_magB_fast_op<32, 8>, sys);
      else
        s = add_gmres_chunks<MagneticBFastOp>(plan, members, mk, F_GMRES_MAG_B, make_magB_fast_op<>, sys);
    }
    else
      s = add_gmres_chunks<MagneticBOp>(plan, members, IMEX_MIXED_MAGNETIC | IMEX_MIXED_MAGNETIC_B, F_GMRES_MAG_B,
                                        make_magB_op, sys);
  } else if (P.formula == IMEX_EnergyFormula) {  // the energy solve, in place on E
    s = add_gmres_chunks<EnergyOp>(plan, members, IMEX_MIXED_PRESSURE, F_GMRES_ENERGY, make_energy_op,
                                   [](imex_ctx* m, double** x, const double** b) {
                                     *x = m->cons + 4 * m->N;
                                     *b = m->pb;
                                   });
  } else if (!P.floor_on && P.eos_type == IMEX_IDEAL_GAS) {  // linear pressure solve
    s = add_gmres_chunks<PressureOp>(plan, members, IMEX_MIXED_PRESSURE, F_NEWTON, make_pressure_op,
                                     [](imex_ctx* m, double** x, const double** b) {
                                       *x = m->pp;
                                       *b = m->pb;
                                     });
  } else if (!mixed(c0, IMEX_MIXED_PRESSURE)) {
    s = add_newton_chunks<double>(plan, members);
  } else {
    s = add_newton_chunks<float>(plan, members);
  }
  if (s != IMEX_OK) {
    batch_solve_free(plan);
    return s;
  }
  *out = plan;
  return IMEX_OK;
}
imex_status batch_solve_run(BatchSolvePlan* plan, cudaStream_t stream, imex_ctx* err_ctx) {
  for (const BatchChunk& ch : plan->chunks) {
    cudaError_t e = ch.launch(stream);
    if (e != cudaSuccess) return cuda_check(err_ctx, e, "batched solve launch");
  }
  return IMEX_OK;
}
void batch_solve_free(BatchSolvePlan* plan) {
  if (!plan) return;
  for (void* p : plan->dev) cudaFree(p);
  delete plan;
}

namespace {
}  // namespace
// gmax_bx / gmax_by from the per-CTA maxima k_stage_combine left in partial
imex_status gmax_finalize(imex_ctx* ctx, int nblk) {
  launch<k_gmax_finalize>(ctx, 1, kGmaxThreads, 0, ctx->stream, ctx->partial, nblk, ctx->sc);
  LAUNCH_CHECK(ctx, "k_gmax_finalize");
  return IMEX_OK;
}
__global__ void k_set_h(DevScalars* sc, double h) { sc->h = h; }
imex_status set_h(imex_ctx* ctx, double h) {
  k_set_h<<<1, 1, 0, ctx->stream>>>(ctx->sc, h);
  LAUNCH_CHECK(ctx, "k_set_h");
  return IMEX_OK;
}
namespace {

}  // namespace

// The magnetic and pressure sub-systems in parts around their solves.  The single-context
// stage runs each part and then its solve; the batched stage runs a part for every member,
// then one batched solve for all of them.

// MagSubsystem_UpdateB (imex_subsystems.cpp:537-628) / MagSubsystem_UpdateA
// (imex_subsystems.cpp:5-74): right-hand side (and the A-form's global viscosity).
imex_status mag_rhs(imex_ctx* ctx) {
  const DevParams& P = ctx->P;
  int nb = blocks_for(P.N);
  imex_status s = local_visc(ctx, mag_visc_mode(ctx));
  if (s != IMEX_OK) return s;
  if (P.magfield == IMEX_PotentialA) {
    if (!ctx->gmax_ready) {  // the stage combination did not take the maxima of this Qs
      int nred = nb < ctx->max_blocks ? nb : ctx->max_blocks;
      prof_begin(ctx);
      launch<k_gmax>(ctx, nred, kThreads, 0, ctx->stream, P, ctx->Qs, ctx->partial);
      LAUNCH_CHECK(ctx, "k_gmax");
      launch<k_gmax_finalize>(ctx, 1, kGmaxThreads, 0, ctx->stream, ctx->partial, nred, ctx->sc);
      LAUNCH_CHECK(ctx, "k_gmax_finalize");
      prof_end(ctx, F_GMAX, BYTES(8), 2);
    }
    ctx->gmax_ready = false;
    prof_begin(ctx);
    launch<k_magnetic_rhs_A>(ctx, nb, kThreads, 0, ctx->stream, P, ctx->sc, ctx->cons, ctx->Qe, ctx->pe, ctx->A_s, ctx->mb,
                             P.fast ? ctx->irho : (double*)nullptr);
    LAUNCH_CHECK(ctx, "k_magnetic_rhs_A");
    prof_end(ctx, F_MAG_RHS, BYTES(P.fast ? 15 : 14), 1);
    return IMEX_OK;
  }
  prof_begin(ctx);
  // the initial guess Qe B goes straight into the cell B planes of u_con (planes 5-7; the
  // kernel reads only planes 0-3 of u_con), which GMRES then overwrites with the solution
  launch<k_magnetic_rhs_B>(ctx, nb, kThreads, 0, ctx->stream, P, ctx->sc, ctx->cons, ctx->Qe, ctx->Qs, ctx->pe, ctx->mb,
                                                    ctx->cons + 5 * P.N);
  LAUNCH_CHECK(ctx, "k_magnetic_rhs_B");
  prof_end(ctx, F_MAG_RHS, BYTES(17), 1);
  return IMEX_OK;
}
// the magnetic system of the current stage: operator, solution (in/out) and right-hand side.
// The A form is solved in place on A (the initial guess is the current A,
// imex_subsystems.cpp:46-60), the B form in the cell B planes of u_con.
void mag_system(imex_ctx* ctx, int* op, double** x, const double** b) {
  const bool a_form = ctx->P.magfield == IMEX_PotentialA;
  *op = a_form ? IMEX_OP_MAGNETIC_A : IMEX_OP_MAGNETIC_B;
  *x = a_form ? ctx->A : ctx->cons + 5 * ctx->P.N;
  *b = ctx->mb;
}
// after the solve: B = curl A, or the face fluxes of the B form (CollectMagFluxes)
imex_status mag_out(imex_ctx* ctx) {
  const DevParams& P = ctx->P;
  int nb = blocks_for(P.N);
  prof_begin(ctx);
  if (P.magfield == IMEX_PotentialA) {
    IMEX_LAUNCH_BC(P, k_curl_A, nb, kThreads, 0, ctx->stream, P, ctx->A, ctx->cons);
    LAUNCH_CHECK(ctx, "k_curl_A");
    prof_end(ctx, F_MAG_OUT, BYTES(6), 1);
  } else {
    launch<k_collect_mag_fluxes>(ctx, nb, kThreads, 0, ctx->stream, P, ctx->sc, ctx->cons, ctx->Qe, ctx->pe, ctx->Fx, ctx->Fy);
    LAUNCH_CHECK(ctx, "k_collect_mag_fluxes");
    prof_end(ctx, F_COLLECT_FLUX, BYTES(12), 1);
  }
  return IMEX_OK;
}
imex_status run_mag_subsystem(imex_ctx* ctx) {
  imex_status s;
  if ((s = mag_rhs(ctx)) != IMEX_OK) return s;
  int op;
  double* x;
  const double* b;
  mag_system(ctx, &op, &x, &b);
  if ((s = gmres_launch(ctx, op, x, b)) != IMEX_OK) return s;
  return mag_out(ctx);
}
imex_status run_mag_subsystem_B(imex_ctx* ctx) { return run_mag_subsystem(ctx); }
imex_status run_mag_subsystem_A(imex_ctx* ctx) { return run_mag_subsystem(ctx); }

// PreSubsystem_Pressure (imex_subsystems.cpp:76-413), DefinitionofU energy, in three
// parts around its one or two nested-Newton solves of p (pp) with right-hand side pb.
imex_status pres_part1(imex_ctx* ctx) {
  const DevParams& P = ctx->P;
  if (P.formula == IMEX_EnergyFormula) return energy_setup(ctx);
  imex_status s;
  if ((s = pressure_setup(ctx)) != IMEX_OK) return s;
  int nb = blocks_for(P.N);
  prof_begin(ctx);
  IMEX_LAUNCH_BC(P, k_pressure_rhs, nb, kThreads, 0, ctx->stream, P, ctx->sc, ctx->cons, ctx->hh, ctx->rv, ctx->rv,
                 ctx->pb, ctx->pe, ctx->pp, P.floor_on ? ctx->sc->bkey[0] : nullptr);
  LAUNCH_CHECK(ctx, "k_pressure_rhs");
  prof_end(ctx, F_PRES_RHS, BYTES(14), 1);
  return IMEX_OK;
}
// momentum from the first solve; *second tells whether a second solve follows
imex_status pres_part2(imex_ctx* ctx, int rks, bool* second) {
  const DevParams& P = ctx->P;
  int nb = blocks_for(P.N);
  if (P.formula == IMEX_EnergyFormula) {
    *second = false;
    return energy_momentum(ctx);
  }
  prof_begin(ctx);
  launch<k_momentum>(ctx, nb, kThreads, 0, ctx->stream, P, ctx->sc, ctx->pp, ctx->rv, ctx->cons);
  LAUNCH_CHECK(ctx, "k_momentum");
  prof_end(ctx, F_MOMENTUM, BYTES(5), 1);
  *second = P.PressureSolver == IMEX_all_correction || (P.PressureSolver == IMEX_once_correction && rks == P.RKs - 1);
  if (*second) {
    prof_begin(ctx);
    IMEX_LAUNCH_BC(P, k_pressure_rhs, nb, kThreads, 0, ctx->stream, P, ctx->sc, ctx->cons, ctx->hh, ctx->rv,
                   ctx->cons + P.N, ctx->pb, nullptr, nullptr, P.floor_on ? ctx->sc->bkey[1] : nullptr);
    LAUNCH_CHECK(ctx, "k_pressure_rhs(2)");
    prof_end(ctx, F_PRES_RHS, BYTES(15), 1);
  }
  return IMEX_OK;
}
imex_status pres_part3(imex_ctx* ctx) {
  const DevParams& P = ctx->P;
  if (P.formula == IMEX_EnergyFormula) return IMEX_OK;
  int nb = blocks_for(P.N);
  prof_begin(ctx);
  if (P.U_update == IMEX_ConservationofU) {
    launch<k_energy_conservation>(ctx, nb, kThreads, 0, ctx->stream, P, ctx->sc, ctx->pp, ctx->cons);
    LAUNCH_CHECK(ctx, "k_energy_conservation");
    prof_end(ctx, F_ENERGY, BYTES(6), 1);  // p, rho, rho vx, rho vy, E in; E out
    return IMEX_OK;
  }
  launch<k_energy_define>(ctx, nb, kThreads, 0, ctx->stream, P, ctx->pp, ctx->cons);
  LAUNCH_CHECK(ctx, "k_energy_define");
  prof_end(ctx, F_ENERGY, BYTES(9), 1);
  return IMEX_OK;
}
imex_status run_pre_subsystem_pressure(imex_ctx* ctx, int rks) {
  imex_status s;
  bool second = false;
  if ((s = pres_part1(ctx)) != IMEX_OK) return s;
  if ((s = newton_launch(ctx, ctx->pp, ctx->pb, 1)) != IMEX_OK) return s;
  if ((s = pres_part2(ctx, rks, &second)) != IMEX_OK) return s;
  if (second && (s = newton_launch(ctx, ctx->pp, ctx->pb, 2)) != IMEX_OK) return s;
  return pres_part3(ctx);
}
// PreSubsystem_Energy (imex_subsystems.cpp:415-534), periodic: one GMRES on E in place
imex_status run_pre_subsystem_energy(imex_ctx* ctx) {
  imex_status s;
  if ((s = energy_setup(ctx)) != IMEX_OK) return s;
  if ((s = gmres_run(ctx, make_energy_op(ctx), F_GMRES_ENERGY, ctx->cons + 4 * ctx->N, ctx->pb,
                     IMEX_MIXED_PRESSURE)) != IMEX_OK)
    return s;
  return energy_momentum(ctx);
}

imex_status prepare_operator(imex_ctx* ctx, int op, double h) {
  imex_status s;
  if (op == IMEX_OP_MAGNETIC_A) {
    const DevParams& P = ctx->P;
    int nred = blocks_for(P.N) < ctx->max_blocks ? blocks_for(P.N) : ctx->max_blocks;
    launch<k_gmax>(ctx, nred, kThreads, 0, ctx->stream, P, ctx->Qs, ctx->partial);
    launch<k_gmax_finalize>(ctx, 1, kGmaxThreads, 0, ctx->stream, ctx->partial, nred, ctx->sc);
    LAUNCH_CHECK(ctx, "k_gmax");
  }
  if ((op == IMEX_OP_MAGNETIC_A || op == IMEX_OP_MAGNETIC_B) &&
      (s = local_visc(ctx, op == IMEX_OP_MAGNETIC_A ? LV_MAG_A : LV_MAG_B)) != IMEX_OK)
    return s;
  if (op == IMEX_OP_MAGNETIC_A && ctx->P.fast) {
    launch<k_recip>(ctx, blocks_for(ctx->P.N), kThreads, 0, ctx->stream, ctx->cons, ctx->irho, ctx->P.N);
    LAUNCH_CHECK(ctx, "k_recip");
  }
  if ((s = set_h(ctx, h)) != IMEX_OK) return s;
  if (op == IMEX_OP_PRESSURE_L || op == IMEX_OP_PRESSURE_J) {
    // the Qe pressure / enthalpy planes come from the stage combination; rebuild them here
    // so that operators can be prepared from externally set buffers too
    if ((s = launch_qe_derived(ctx)) != IMEX_OK) return s;
    return pressure_setup(ctx);
  }
  if (op == IMEX_OP_ENERGY) return energy_setup(ctx);
  return IMEX_OK;
}

imex_status set_newton_state(imex_ctx* ctx, const double* pf, double mbig) {
  // vdiag = V_slope(p_freeze, rho) with the given Mbig
  cudaError_t e = cudaMemcpyAsync(ctx->pf, pf, ctx->N * sizeof(double), cudaMemcpyDefault, ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "p_freeze upload");
  ctx->h_sc->Mbig = mbig;
  e = cudaMemcpyAsync(&ctx->sc->Mbig, &ctx->h_sc->Mbig, sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "Mbig upload");
  return launch_vslope(ctx);
}

imex_status apply_operator(imex_ctx* ctx, int op, const double* x, double* Ax) {
  Tiling T = make_tiling(ctx->nx, ctx->ny, ctx->P.xclamp, ctx->P.yclamp);
  int nb = T.ntiles < ctx->max_blocks ? T.ntiles : ctx->max_blocks;
  if (op == IMEX_OP_PRESSURE_L || op == IMEX_OP_PRESSURE_J) {
    PressureOp o = make_pressure_op(ctx);
    o.jac = op == IMEX_OP_PRESSURE_J;
    launch_apply(ctx, o, nb, T, x, Ax);
  } else if (op == IMEX_OP_MAGNETIC_B) {
    if (ctx->P.fast) launch_apply(ctx, make_magB_fast_op<>(ctx), nb, T, x, Ax);
    else launch_apply(ctx, make_magB_op(ctx), nb, T, x, Ax);
  } else if (op == IMEX_OP_MAGNETIC_A) {
    if (ctx->P.xclamp || ctx->P.yclamp) launch_apply(ctx, make_magA_op<true>(ctx), nb, T, x, Ax);
    else launch_apply(ctx, make_magA_op(ctx), nb, T, x, Ax);
  } else if (op == IMEX_OP_ENERGY) {
    launch_apply(ctx, make_energy_op(ctx), nb, T, x, Ax);
  } else {
    return set_error(ctx, IMEX_ERR_UNSUPPORTED, "operator not available");
  }
  LAUNCH_CHECK(ctx, "k_apply");
  return IMEX_OK;
}

imex_status run_gmres(imex_ctx* ctx, int op, double* x, const double* b) { return gmres_launch(ctx, op, x, b); }

imex_status run_gmres_noalloc(imex_ctx* ctx, int op, double* x, const double* b, unsigned char* base,
                              size_t capacity) {
  if (op == IMEX_OP_PRESSURE_L || op == IMEX_OP_PRESSURE_J) {
    PressureOp o = make_pressure_op(ctx);
    o.jac = op == IMEX_OP_PRESSURE_J;
    return gmres_noalloc_op(ctx, o, F_GMRES_PRES, x, b, base, capacity);
  } else if (op == IMEX_OP_MAGNETIC_B) {
    return gmres_noalloc_op(ctx, make_magB_op(ctx), F_GMRES_MAG_B, x, b, base, capacity);
  } else if (op == IMEX_OP_MAGNETIC_A) {
    if (ctx->P.xclamp || ctx->P.yclamp)
      return gmres_noalloc_op(ctx, make_magA_op<true>(ctx), F_GMRES_MAG_A, x, b, base, capacity);
    return gmres_noalloc_op(ctx, make_magA_op(ctx), F_GMRES_MAG_A, x, b, base, capacity);
  } else if (op == IMEX_OP_ENERGY) {
    return gmres_noalloc_op(ctx, make_energy_op(ctx), F_GMRES_ENERGY, x, b, base, capacity);
  }
  return set_error(ctx, IMEX_ERR_UNSUPPORTED, "operator not available");
}

imex_status run_barrier_selftest(imex_ctx* ctx, int iterations, int phantom_blocks, double timeout_s,
                                 double* us_per_barrier) {
  const Tiling T = make_tiling(ctx->nx, ctx->ny, ctx->P.xclamp, ctx->P.yclamp);
  int nb = coop_blocks<MagneticAOp>(ctx, (const void*)k_gmres<MagneticAOp>, T);
  const double saved = ctx->barrier_timeout_s;
  ctx->barrier_timeout_s = timeout_s;
  imex_status s = reset_sync(ctx);
  ctx->barrier_timeout_s = saved;
  if (s != IMEX_OK) return s;
  long long* cyc = reinterpret_cast<long long*>(ctx->red);
  unsigned phantom = (unsigned)(phantom_blocks > 0 ? phantom_blocks : 0);
  void* params[] = {(void*)&ctx->sync, (void*)&phantom, (void*)&iterations, (void*)&ctx->st, (void*)&cyc};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_barrier_selftest, dim3(nb), dim3(NT), params, 0,
                                              ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "barrier self-test launch");
  long long h = 0;
  e = cudaMemcpyAsync(&h, cyc, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "barrier self-test");
  const int clk_khz = ctx->clock_khz;
  if (us_per_barrier) *us_per_barrier = (iterations > 0 && clk_khz > 0) ? (double)h / iterations / (clk_khz * 1e-3) : 0.0;
  return IMEX_OK;
}
imex_status run_nested_newton(imex_ctx* ctx, double* p, const double* b) { return newton_launch(ctx, p, b); }


// ================================================================== adjoint building blocks
// The operators evaluated on the 3x3 local tile of one cell, through the same tile-buffer
// interface the solver kernels stage (halo 1), in any scalar type: with Dual<L> they give
// columns of the operator's stencil (transposed solves) or of its dependence on the frozen
// coefficients (coefficient adjoints).
namespace {
template <class Op, class T>
struct LocalTile {
  static constexpr int SX = 3, SY = 3, SN = 9;
  T s[Op::M * SN];
  T c[(Op::QT > 0 ? Op::QT : 1) * SN];
  T p[1];
};
// coefficients of the nine cells around nb[4]; the vector from x (planes of N) or zero
template <class Op, class T>
__device__ __forceinline__ void local_fill(const Op& od, LocalTile<Op, T>& t, const long long* nb, const double* x,
                                           long long N) {
  constexpr int QC = Op::QT > 0 ? Op::QT : 1;
  for (int q = 0; q < 9; ++q) {
    T cq[QC];
    od.coef(nb[q], cq);
    for (int k = 0; k < Op::QT; ++k) t.c[k * 9 + q] = cq[k];
    for (int k = 0; k < Op::M; ++k) t.s[k * 9 + q] = x ? T(x[k * N + nb[q]]) : T(0.0);
  }
}
// viscosity scalars of the operators (cx, cy: magnetic; cvx, cvy: pressure)
__device__ __forceinline__ void set_visc(MagneticBCoef& c, double a, double b) {
  c.cx = a;
  c.cy = b;
}
__device__ __forceinline__ void set_visc(PressureCoef& c, double a, double b) {
  c.cvx = a;
  c.cvy = b;
}

// Transposed stencil of a linear operator: AT[(o M + k') M + k] at cell c' = c + offset(o)
// holds d(A x)[k](c) / d x[k'](c'), so (A^T mu)[k'](c') = sum_o sum_k AT[..](c') mu[k](c' - o).
template <class Op>
__global__ void k_adj_assemble_T(Op op, DevParams P, double* __restrict__ AT) {
  constexpr int M = Op::M;
  using D = Dual<M>;
  const long long N = P.N;
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  op.bind();
  const auto od = op.template as<D>();
  using OD = typename std::remove_const<decltype(od)>::type;
  long long nb[9];
  neighbours(P, n, nb);
  LocalTile<OD, D> t;
  local_fill(od, t, nb, nullptr, N);
  for (int o = 0; o < 9; ++o) {
    for (int kk = 0; kk < M; ++kk) t.s[kk * 9 + o].d[kk] = 1.0;
    D out[M];
    od.matvec(t, 0, 0, n, out);
    for (int kk = 0; kk < M; ++kk)
      for (int k = 0; k < M; ++k) AT[((long long)(o * M + kk) * M + k) * N + nb[o]] = out[k].d[kk];
    for (int kk = 0; kk < M; ++kk) t.s[kk * 9 + o].d[kk] = 0.0;
  }
}

// The assembled transposed operator in the solver-kernel interface (FP64 only), with the
// Jacobi preconditioner of its diagonal.
template <int M_>
struct AssembledTOp {
  using value_type = double;
  static constexpr int M = M_, HALO = 1;
  static constexpr int COEF = 9 * M_ * M_;
  static constexpr int QT = 1;  // nothing staged; one dummy plane keeps the tile layout
  static constexpr int PT = 0;
  static constexpr int MIN_BLOCKS = 2;
  const double* AT;
  long long N;
  __device__ __forceinline__ void bind() {}
  template <class U>
  __device__ __forceinline__ AssembledTOp as() const {
    return *this;
  }
  __device__ __forceinline__ void coef(long long, double* q) const { q[0] = 0.0; }
  template <class TB>
  __device__ __forceinline__ void prepass(TB&, int, int) const {}
  template <class TB>
  __device__ __forceinline__ void matvec(const TB& tb, int lx, int ly, long long c, double* out) const {
    const int o0 = (ly + 1) * TB::SX + lx + 1;
#pragma unroll
    for (int kk = 0; kk < M; ++kk) out[kk] = 0.0;
#pragma unroll
    for (int o = 0; o < 9; ++o) {
      const int src = o0 - (o % 3 - 1) - (o / 3 - 1) * TB::SX;
#pragma unroll
      for (int kk = 0; kk < M; ++kk)
#pragma unroll
        for (int k = 0; k < M; ++k) out[kk] += __ldg(AT + ((long long)(o * M + kk) * M + k) * N + c) * tb.s[k * TB::SN + src];
    }
  }
  __device__ __forceinline__ void precond(long long c, double* v) const {
#pragma unroll
    for (int k = 0; k < M; ++k) v[k] = v[k] / __ldg(AT + ((long long)(4 * M + k) * M + k) * N + c);
  }
};

// coefficient adjoint: lam_q(c + o) -= sum_k mu[k](c) d(A x)[k](c) / d coef_q(c + o), at fixed x
struct LamPlanes {
  double* p[4];
};
template <class Op>
__global__ void k_adj_coef_vjp(Op op, DevParams P, const double* __restrict__ x, const double* __restrict__ mu,
                               LamPlanes lam) {
  constexpr int M = Op::M, QT = Op::QT;
  using D = Dual<QT>;
  const long long N = P.N;
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  op.bind();
  const auto od = op.template as<D>();
  using OD = typename std::remove_const<decltype(od)>::type;
  long long nb[9];
  neighbours(P, n, nb);
  LocalTile<OD, D> t;
  local_fill(od, t, nb, x, N);
  double m[M];
  for (int k = 0; k < M; ++k) m[k] = mu[k * N + n];
  for (int o = 0; o < 9; ++o) {
    for (int q = 0; q < QT; ++q) t.c[q * 9 + o].d[q] = 1.0;
    D out[M];
    od.matvec(t, 0, 0, n, out);
    for (int q = 0; q < QT; ++q) {
      double s = 0.0;
      for (int k = 0; k < M; ++k) s += m[k] * out[k].d[q];
      if (s != 0.0 && lam.p[q]) atomicAdd(lam.p[q] + nb[o], -s);
    }
    for (int q = 0; q < QT; ++q) t.c[q * 9 + o].d[q] = 0.0;
  }
}
// viscosity-scalar adjoint: the operators are affine in their two viscosity scalars, so
// d(A x)/d c = A x |(c=1) - A x |(c=0); lam2[0..1] -= sum_cells mu . d(A x)/d c
template <class Op>
__global__ void k_adj_visc_vjp(Op op, DevParams P, const double* __restrict__ x, const double* __restrict__ mu,
                               double* __restrict__ lam2) {
  constexpr int M = Op::M;
  const long long N = P.N;
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double sx = 0.0, sy = 0.0;
  if (n < N) {
    op.bind();
    long long nb[9];
    neighbours(P, n, nb);
    LocalTile<Op, double> t;
    local_fill(op, t, nb, x, N);
    Op o0 = op, ox = op, oy = op;
    set_visc(o0, 0.0, 0.0);
    set_visc(ox, 1.0, 0.0);
    set_visc(oy, 0.0, 1.0);
    double a0[M], ax[M], ay[M];
    o0.matvec(t, 0, 0, n, a0);
    ox.matvec(t, 0, 0, n, ax);
    oy.matvec(t, 0, 0, n, ay);
    for (int k = 0; k < M; ++k) {
      const double m = mu[k * N + n];
      sx += m * (ax[k] - a0[k]);
      sy += m * (ay[k] - a0[k]);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (sx != 0.0) atomicAdd(lam2, -sx);
    if (sy != 0.0) atomicAdd(lam2 + 1, -sy);
  }
}

template <class Op>
imex_status adj_op_dispatch(imex_ctx* ctx, const AdjOp& a, Op* out);
template <>
imex_status adj_op_dispatch(imex_ctx* ctx, const AdjOp& a, MagneticBOp* out) {
  MagneticBOp o = make_magB_op(ctx);
  o.Qe = a.Qe;
  o.rho = a.rho;
  *out = o;
  return IMEX_OK;
}
template <>
imex_status adj_op_dispatch(imex_ctx* ctx, const AdjOp& a, PressureOp* out) {
  PressureOp o = make_pressure_op(ctx);
  o.hh = a.hh;
  o.eta = a.eta;
  o.rho = a.rho;
  o.vscale = a.vscale;
  o.vdiag = a.vdiag;
  o.jac = a.kind == ADJ_OP_PRESSURE_J;
  *out = o;
  return IMEX_OK;
}

template <class Op, int M>
imex_status adj_transpose_solve_op(imex_ctx* ctx, const AdjOp& a, double* AT, double* mu, const double* lam,
                                   double tol) {
  Op op;
  adj_op_dispatch(ctx, a, &op);
  const DevParams& P = ctx->P;
  const int nb = blocks_for(P.N);
  prof_begin(ctx);
  k_adj_assemble_T<Op><<<nb, kThreads, 0, ctx->stream>>>(op, P, AT);
  LAUNCH_CHECK(ctx, "k_adj_assemble_T");
  prof_end(ctx, F_ADJ_ASSEMBLE, 0.0, 1);
  cudaError_t e = cudaMemsetAsync(mu, 0, (size_t)M * P.N * sizeof(double), ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "adjoint initial guess");
  AssembledTOp<M> T{};
  T.AT = AT;
  T.N = P.N;
  const Tiling TL = make_tiling(ctx->nx, ctx->ny, ctx->P.xclamp, ctx->P.yclamp);
  auto kern = k_gmres<AssembledTOp<M>>;
  const int nblk = coop_blocks<AssembledTOp<M>>(ctx, (const void*)kern, TL);
  GmresWork g = make_work(ctx, TL, nblk, F_ADJOINT);
  g.tol = tol;
  g.tol_abs = 0.0;
  prof_begin(ctx);
  imex_status s = launch_coop<AssembledTOp<M>>(ctx, kern, nblk, T, g, mu, lam);
  prof_end(ctx, F_ADJOINT, 0.0, 2);
  return s;
}
template <class Op>
imex_status adj_coef_vjp_op(imex_ctx* ctx, const AdjOp& a, const double* x, const double* mu, double* const* lam_q,
                            double* lam_visc) {
  Op op;
  adj_op_dispatch(ctx, a, &op);
  const DevParams& P = ctx->P;
  const int nb = blocks_for(P.N);
  LamPlanes L{};
  for (int q = 0; q < Op::QT && q < 4; ++q) L.p[q] = lam_q[q];
  prof_begin(ctx);
  k_adj_coef_vjp<Op><<<nb, kThreads, 0, ctx->stream>>>(op, P, x, mu, L);
  LAUNCH_CHECK(ctx, "k_adj_coef_vjp");
  if (lam_visc) {
    k_adj_visc_vjp<Op><<<nb, kThreads, 0, ctx->stream>>>(op, P, x, mu, lam_visc);
    LAUNCH_CHECK(ctx, "k_adj_visc_vjp");
  }
  prof_end(ctx, F_ADJ_ASSEMBLE, 0.0, lam_visc ? 2 : 1);
  return IMEX_OK;
}
}  // namespace

imex_status adj_transpose_solve(imex_ctx* ctx, const AdjOp& a, double* AT, double* mu, const double* lam, double tol) {
  if (a.kind == ADJ_OP_MAGNETIC_B) return adj_transpose_solve_op<MagneticBOp, 3>(ctx, a, AT, mu, lam, tol);
  return adj_transpose_solve_op<PressureOp, 1>(ctx, a, AT, mu, lam, tol);
}
imex_status adj_coef_vjp(imex_ctx* ctx, const AdjOp& a, const double* x, const double* mu, double* const* lam_q,
                         double* lam_visc) {
  if (a.kind == ADJ_OP_MAGNETIC_B) return adj_coef_vjp_op<MagneticBOp>(ctx, a, x, mu, lam_q, lam_visc);
  return adj_coef_vjp_op<PressureOp>(ctx, a, x, mu, lam_q, lam_visc);
}
imex_status adj_apply(imex_ctx* ctx, const AdjOp& a, const double* x, double* Ax) {
  Tiling T = make_tiling(ctx->nx, ctx->ny, ctx->P.xclamp, ctx->P.yclamp);
  int nb = T.ntiles < ctx->max_blocks ? T.ntiles : ctx->max_blocks;
  if (a.kind == ADJ_OP_MAGNETIC_B) {
    MagneticBOp o;
    adj_op_dispatch(ctx, a, &o);
    launch_apply(ctx, o, nb, T, x, Ax);
  } else {
    PressureOp o;
    adj_op_dispatch(ctx, a, &o);
    launch_apply(ctx, o, nb, T, x, Ax);
  }
  LAUNCH_CHECK(ctx, "k_apply");
  return IMEX_OK;
}

// queue the copy of this translation unit's EOS flag into pinned host memory (no wait)
imex_status eos_flag_solve_enqueue(imex_ctx* ctx, int* host_flag) {
  return cuda_check(ctx, cudaMemcpyFromSymbolAsync(host_flag, d_eos_flag, sizeof(int), 0, cudaMemcpyDeviceToHost,
                                                   ctx->stream),
                    "eos flag");
}
imex_status eos_flag_solve(imex_ctx* ctx, int* flag, bool reset) {
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
