// Internal declarations shared by the CUDA sources of libimex_b200.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <functional>
#include <string>
#include <vector>

#include "../../include/imex_b200.h"

namespace imex {

struct Recorder;  // launch.cuh: the recorded launches of a context while an ensemble plans a step

constexpr int kMaxRK = 3;
constexpr int kMaxKrylov = 32;  // upper bound on gmres_restart (reference: 25)

// Solver constants of one context, passed to kernels by value.
struct DevParams {
  int nx, ny;
  long long N;  // nx * ny
  double dx, dy, hmin;
  int formula, magfield, recon, reconstate, vortex_minmod, GLF, add_bvisc, add_pvisc;
  int U_update, PressureSolver, Energy_Modify, floor_on, Pnewton_max, eos_type, caltimestep, RKs;
  double gamma, m_alfa, m_b, m_R, m_cv;
  double p_floor, Mbig_fac, theta, Pnewton_tol, shock_kappa1, GMREStol, CFL, time_stop, fixed_dt;
  // 1 where the direction is transmissive: neighbour indices clamp to the nearest interior
  // cell (bound_cond_u / bound_cond_array / M_P / M_B, boundary.cpp:7-16,
  // timestep.cpp:168-204, implicit_operators.cpp:12-14); 0 where it is periodic (wrap)
  int xclamp, yclamp;
  // the index map as one multiply-add per side: i < 0 -> i * xm + xlo, i >= nx -> i * xm + xhi
  // (periodic: xm = 1, xlo = nx, xhi = -nx; transmissive: xm = 0, xlo = 0, xhi = nx - 1)
  int xm, xlo, xhi, ym, ylo, yhi;
  int fast;  // imex_config.arith == IMEX_ARITH_FAST (explicit stencil kernels)
  // division of a cell index by nx as a multiply-high and two shifts (cell_of): the magic
  // number and shifts of Granlund and Montgomery's division by an invariant integer
  unsigned nx_magic;
  int nx_sh1, nx_sh2;
  // 1 / dx and 1 / dy, divided once on the host (both sides round the quotient to nearest, so
  // a kernel reading them gets the value its own 1.0 / dx would give)
  double rdx, rdy;
};

// Boundary normal faces of the transmissive directions.  The reference keeps Bx_p0 at
// x = x_0 and By_0p at y = y_0 as degrees of freedom that CT evolves and that the cell
// average of the first row / column reads (constrained_transport.cpp:5-30,
// ct_flux.cpp:176-189); a periodic direction identifies them with the faces at x_1 / y_1.
// One line of ny values per Bx array, nx per By array; ex / ey hold the corner EMFs on
// x = x_0 (corners j - 1/2 for j = 0..ny) and on y = y_0 (corners i - 1/2 for i = 0..nx).
struct BoundaryLines {
  double *bx, *bx_n, *bxQe, *bxQs, *hsbx;  // hsbx: RKs lines (the HsB of each stage)
  double *by, *by_n, *byQe, *byQs, *hsby;
  double *ex, *ey;
};

// Scalars living in device memory (the reference's hidden globals).
struct DevScalars {
  double dt, adt, B_max_x, B_max_y, vx_max, vy_max, v_max, a_max;
  double ch, ch_x, ch_y, cA, cA_x, cA_y, t, prev_dt, Mbig;
  double gmax_bx, gmax_by;  // A-form viscosity maxima of the current solve
  double h;                 // implicit step of the current sub-step
  int timestep;
  int pad;
  // order keys (dkey) of min b and of ~max V(p_floor, rho) over the cells, from the pressure
  // right-hand sides of a stage (slot 0: the first solve, slot 1: the second) for the nested
  // Newton's floor slope Mbig; k_pressure_coeffs resets them at the start of the sub-system
  unsigned long long bkey[2][2];
};

// Kernel launch families of the live profile.
enum Family {
  F_PROLOGUE_REDUCE, F_CONS_FROM_PRIM, F_COMBINE, F_RECON, F_FLUX_CONV, F_FLUX_PRES, F_MAG_RHS,
  F_GMRES_MAG_B, F_GMRES_MAG_A, F_MAG_OUT, F_COLLECT_FLUX, F_PRES_SETUP, F_SHOCK, F_PRES_RHS, F_NEWTON,
  F_MOMENTUM, F_ENERGY, F_CT, F_DERIVATIVE, F_GMAX, F_GMRES_PRES, F_APPLY, F_MIXED, F_GMRES_ENERGY, F_ADJOINT, F_ADJ_CELLS, F_ADJ_FLUX, F_ADJ_LINEAR, F_ADJ_ASSEMBLE, NFAM
};

// Device-side counters and status of the implicit solves.
struct DevStats {
  int gmres_solves, gmres_iters, gmres_restarts, newton_iters, max_floored, refine_sweeps;
  int status;      // worst imex_status
  int barrier_fail;
  double last_residual, min_p;
  double alg_bytes[NFAM];  // algorithmic bytes counted by the persistent kernels
};

// Host-side event profiler of launch families.
struct ProfRec {
  cudaEvent_t a, b;
  int fam;
  double bytes;
};

// Grid-barrier and reduction workspace of the persistent solver kernels.
struct SyncState {
  unsigned long long count;  // barrier arrivals since the launch started (monotonic, 64-bit: never wraps)
  int abort;
  int pad1;
  long long wait_cycles;  // bound of any single barrier wait, in SM clock cycles
};

}  // namespace imex

struct imex_ctx {
  imex_config cfg{};
  imex::DevParams P{};
  int nx = 0, ny = 0;
  size_t N = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string last_error;
  int num_sms = 0;
  int clock_khz = 0;  // maximum SM clock, read once at creation (bounds of device-side waits)
  int device = -1;    // the device that was current at imex_create; all its memory lives there
  bool keep_shock_chit = false;  // the shock detector also stores chi~ in chit (the adjoint reads it)

  // device state (interior planes)
  double *prim = nullptr, *cons = nullptr, *cons_n = nullptr, *Qe = nullptr, *Qs = nullptr;
  double *bx = nullptr, *by = nullptr, *bx_n = nullptr, *by_n = nullptr, *bxQe = nullptr, *byQe = nullptr;
  double *bxQs = nullptr, *byQs = nullptr, *Fx = nullptr, *Fy = nullptr;
  double *A = nullptr, *A_s = nullptr, *A_e = nullptr, *A_snap = nullptr;
  double *Hs = nullptr, *HsA = nullptr, *HsB = nullptr, *w = nullptr, *Bsave = nullptr;
  // per-stage derived planes
  double *pe = nullptr;    // pressure of Qe
  double *hQe = nullptr;   // enthalpy e + p/rho of Qe
  // implicit-solve planes
  double *hh = nullptr, *eta = nullptr, *vscale = nullptr, *tdiag = nullptr, *vdiag = nullptr;
  double* irho = nullptr;  // fast arithmetic: 1/rho of u_con for the A-form operator
  double *rv = nullptr;    // rho v* snapshot (3 planes)
  // local Lax-Friedrichs face viscosities (GLF off, else null), 4 planes each: the magnetic
  // operator's and the pressure operator's, built before their solves (k_local_visc)
  double *lvm = nullptr, *lvp = nullptr;
  double *pb = nullptr, *pp = nullptr, *pf = nullptr, *pg = nullptr, *pdp = nullptr;  // pressure vectors
  double *mx = nullptr, *mb = nullptr;  // magnetic solution / rhs (3 planes each)
  double *chit = nullptr, *Epp = nullptr, *Et = nullptr;
  double* bline = nullptr;  // storage of the boundary lines
  imex::BoundaryLines bl{};
  // GMRES workspace
  double* V = nullptr;      // (restart + 1) * 3 planes
  double* AV = nullptr;     // 2 * 3 planes
  double* partial = nullptr;
  long long partial_len = 0;  // doubles in partial
  int max_blocks = 0;
  bool gmax_ready = false;  // gmax_bx / gmax_by already hold the maxima of the current Qs
  float* Vf = nullptr;      // FP32 basis (mixed precision)
  float* AVf = nullptr;
  double* mres = nullptr;   // refinement residual (3 planes)
  double* mcor = nullptr;   // refinement correction (3 planes)
  // scalars and stats
  imex::DevScalars* sc = nullptr;
  imex::DevStats* st = nullptr;
  imex::SyncState* sync = nullptr;
  imex::DevScalars* h_sc = nullptr;  // pinned mirrors
  imex::DevStats* h_st = nullptr;
  double* red = nullptr;    // small reduction buffer (device)
  double* h_red = nullptr;  // pinned mirror
  std::vector<void*> allocations;
  // live profile
  bool prof_on = false;
  std::vector<imex::ProfRec> prof_pending;
  std::vector<cudaEvent_t> prof_pool;
  double prof_ms[imex::NFAM] = {};
  double prof_bytes[imex::NFAM] = {};
  long long prof_launches[imex::NFAM] = {};
  cudaEvent_t prof_open = nullptr;
  long long kernel_launches = 0;  // every kernel this context launched
  imex::Recorder* rec = nullptr;  // set while an ensemble records this context's launches
  double barrier_timeout_s = 2.0;  // bound on any single device-wide wait
};

// Launch (or record, launch.cuh) kernel body kern<kOpen> with the instance for this
// context's boundaries (bc_params): transmissive in x or y, or periodic in both.  The
// calling function's `ctx` is the context that launches.
#define IMEX_LAUNCH_BC(P, kern, grid, block, smem, stream, ...)                         \
  do {                                                                                  \
    if ((P).xclamp || (P).yclamp) launch<kern<true>>(ctx, grid, block, smem, stream, __VA_ARGS__); \
    else launch<kern<false>>(ctx, grid, block, smem, stream, __VA_ARGS__);              \
  } while (0)
// the same over the boundary kind and the arithmetic of the explicit stencils (kern<kOpen, kFast>)
#define IMEX_LAUNCH_BC_ARITH(P, kern, grid, block, smem, stream, ...)                                    \
  do {                                                                                                   \
    const bool open_ = (P).xclamp || (P).yclamp;                                                         \
    if (open_ && (P).fast) launch<kern<true, true>>(ctx, grid, block, smem, stream, __VA_ARGS__);         \
    else if (open_) launch<kern<true, false>>(ctx, grid, block, smem, stream, __VA_ARGS__);              \
    else if ((P).fast) launch<kern<false, true>>(ctx, grid, block, smem, stream, __VA_ARGS__);           \
    else launch<kern<false, false>>(ctx, grid, block, smem, stream, __VA_ARGS__);                        \
  } while (0)

namespace imex {

// live profile: bracket a launch family with events (no-ops when profiling is off)
void prof_begin(imex_ctx* ctx);
void prof_end(imex_ctx* ctx, int fam, double bytes, int kernels);
void prof_harvest(imex_ctx* ctx);
const char* family_name(int fam);

// error helpers
imex_status set_error(imex_ctx* ctx, imex_status s, const std::string& msg);
imex_status cuda_check(imex_ctx* ctx, cudaError_t e, const char* what);

// launchers implemented in kernels_stage.cu
imex_status launch_step_prologue(imex_ctx* ctx);
imex_status launch_stage_combine(imex_ctx* ctx, int rks);
imex_status gmax_finalize(imex_ctx* ctx, int nblk);
imex_status launch_reconstruct(imex_ctx* ctx, bool full);
imex_status launch_flux_update(imex_ctx* ctx, int form);
int second_flux_form(const imex_ctx* ctx);
imex_status launch_stage_derivative(imex_ctx* ctx, int rks);
imex_status launch_ct(imex_ctx* ctx, int variant);
imex_status launch_prim_from_cons(imex_ctx* ctx);
imex_status launch_cons_from_prim(imex_ctx* ctx);
imex_status launch_shock(imex_ctx* ctx, const double* Q, double* eta);
imex_status launch_divergence(imex_ctx* ctx, double* out4);
imex_status launch_ct_diag(imex_ctx* ctx, double* out16);
imex_status launch_min_pressure(imex_ctx* ctx, double* pmin);
imex_status launch_qe_derived(imex_ctx* ctx);
imex_status launch_vslope(imex_ctx* ctx);
// Butcher tableaux Ae, Ai of the IMEX-RK scheme (main.cpp:269-319)
void tableau(int RKs, double ae[kMaxRK][kMaxRK], double ai[kMaxRK][kMaxRK]);

// launchers implemented in kernels_solve.cu
// the implicit step h of these sub-steps is read from device scalars (set_h or the stage combination)
imex_status set_h(imex_ctx* ctx, double h);
imex_status run_mag_subsystem_B(imex_ctx* ctx);
imex_status run_mag_subsystem_A(imex_ctx* ctx);
imex_status run_pre_subsystem_pressure(imex_ctx* ctx, int rks);
imex_status run_pre_subsystem_energy(imex_ctx* ctx);
// the same sub-systems in parts around their solves (the batched stage drives these); in the
// energy formula the pres_part* functions run PreSubsystem_Energy around its one solve
imex_status mag_rhs(imex_ctx* ctx);
void mag_system(imex_ctx* ctx, int* op, double** x, const double** b);
imex_status mag_out(imex_ctx* ctx);
imex_status pres_part1(imex_ctx* ctx);
imex_status pres_part2(imex_ctx* ctx, int rks, bool* second);
imex_status pres_part3(imex_ctx* ctx);
imex_status prepare_operator(imex_ctx* ctx, int op, double h);
imex_status apply_operator(imex_ctx* ctx, int op, const double* x, double* Ax);
imex_status run_gmres(imex_ctx* ctx, int op, double* x, const double* b);
imex_status run_nested_newton(imex_ctx* ctx, double* p, const double* b);
imex_status set_newton_state(imex_ctx* ctx, const double* pf, double mbig);
imex_status run_fp64_selftest(imex_ctx* ctx, double* dfma_per_s, double* ddiv_per_s);
imex_status run_barrier_selftest(imex_ctx* ctx, int iterations, int phantom_blocks, double timeout_s,
                                 double* us_per_barrier);

// batched solves of an ensemble (kernels_solve.cu): one kind of solve for every member, run
// as cooperative launches in which each member owns a contiguous range of CTAs
enum { BATCH_MAGNETIC = 0, BATCH_PRESSURE = 1 };
struct BatchChunk {
  std::function<cudaError_t(cudaStream_t)> launch;  // barrier reset + the cooperative launch
  int ctas = 0, members = 0;
};
struct BatchSolvePlan {
  std::vector<BatchChunk> chunks;
  std::vector<void*> dev;  // device arrays of the plan (jobs, CTA map, barrier pointers)
};
// tile: the shape of the B-form magnetic solve's tiles in the fast arithmetic (kBatchTiles)
imex_status batch_solve_build(const std::vector<imex_ctx*>& members, int kind, BatchSolvePlan** out, int tile = 0);
// the solve tile shapes an ensemble can choose: cells in x and y of tile 0, 1, 2 (64 x 16
// tiles were measured too: 1.2 KB of spills at 128 registers, 1.8x slower)
constexpr int kBatchTiles = 3;
constexpr int kBatchTileX[kBatchTiles] = {32, 64, 32}, kBatchTileY[kBatchTiles] = {16, 8, 8};
imex_status batch_solve_run(BatchSolvePlan* plan, cudaStream_t stream, imex_ctx* err_ctx);
void batch_solve_free(BatchSolvePlan* plan);

// adjoint building blocks (kernels_solve.cu): the operators of one solve on explicit planes
enum { ADJ_OP_PRESSURE_L = 0, ADJ_OP_PRESSURE_J = 1, ADJ_OP_MAGNETIC_B = 2 };
struct AdjOp {
  int kind;
  const double *Qe, *rho;                  // magnetic B: Qe (8 planes), rho (one plane)
  const double *hh, *eta, *vscale, *vdiag;  // pressure (vdiag: J mode)
};
// mu = A^{-T} lam by GMRES on the assembled transposed stencil AT (9 M^2 planes of scratch)
imex_status adj_transpose_solve(imex_ctx* ctx, const AdjOp& a, double* AT, double* mu, const double* lam, double tol);
// lam_q[q](cells) -= mu^T d(A x)/d coef_q for the staged coefficients (magnetic B: Qe Bx, By,
// Bz, rho; pressure: hh, eta) and, if lam_visc, lam_visc[0..1] -= mu^T d(A x)/d (viscosity scalars)
imex_status adj_coef_vjp(imex_ctx* ctx, const AdjOp& a, const double* x, const double* mu, double* const* lam_q,
                         double* lam_visc);
imex_status adj_apply(imex_ctx* ctx, const AdjOp& a, const double* x, double* Ax);

// fixed device scratch of imex_gmres_noalloc (noalloc.cu) and the solve that uses it
constexpr size_t kStaticScratchBytes = IMEX_NOALLOC_SCRATCH_BYTES;
imex_status static_scratch(imex_ctx* ctx, unsigned char** base);
void forget_static_scratch(int dev);  // drop the cached address (imex_create)
imex_status run_gmres_noalloc(imex_ctx* ctx, int op, double* x, const double* b, unsigned char* base,
                              size_t capacity);

}  // namespace imex
