/*
 * imex_b200 - one IMEX Runge-Kutta stage of the 2D ideal-MHD scheme of the
 * IMEX reference solver, as hand-written CUDA for B200 (sm_100a).
 *
 * This header is the whole drop-in boundary: plain C, plain pointers and
 * sizes.  Each entry point replaces one function of the reference's C++
 * interface (include/declarations.hpp) or one block of its driver
 * (src/main.cpp); the citation is given beside it.  A time-marching driver
 * that used to call the reference's sub-system functions calls these in the
 * same order.
 *
 * Data layout exchanged through the interface (host or device pointers are
 * both accepted wherever an array is passed; copies use cudaMemcpyDefault):
 *   - a "plane" is nx*ny doubles of interior cells, index i + nx*j;
 *   - cell state = 8 planes: rho, rho vx, rho vy, rho vz, E, Bx, By, Bz
 *     (conserved) or rho, vx, vy, vz, p, Bx, By, Bz (primitive);
 *   - face fields: plane(i,j) is Bx at the x-face (i+1/2, j), resp. By at the
 *     y-face (i, j+1/2);
 *   - vector potential = 3 planes (Ax, Ay, Az) at cell centres;
 *   - a GMRES vector of the pressure system is one plane; of the magnetic
 *     systems three planes, in the order of the reference's M_P / M_B maps
 *     (implicit_operators.cpp:5-139).
 * Ghost cells do not exist: each direction is periodic or transmissive
 * (imex_config.x_bc / y_bc), and the kernels read a neighbour past the edge
 * through an index map (wrap-around for periodic, the nearest interior cell
 * for transmissive).  The boundary normal faces of a transmissive direction
 * are extra degrees of freedom (imex_set_boundary_faces).
 *
 * Conventions: every function returns imex_status (0 = OK).  Non-convergence
 * and non-finite values found on the device are reported through the status
 * and imex_solve_stats, never by trapping the GPU.  The context owns all
 * device memory.  One context must not be used by two host threads at once.
 * Work is enqueued on the context's stream (imex_set_stream); functions that
 * return results to host memory synchronise that stream.
 */
#ifndef IMEX_B200_H
#define IMEX_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum imex_status {
  IMEX_OK = 0,
  IMEX_ERR_INVALID = 1,     /* bad argument, size or call order */
  IMEX_ERR_UNSUPPORTED = 2, /* configuration this implementation does not cover */
  IMEX_ERR_CUDA = 3,        /* a CUDA runtime call failed */
  IMEX_GMRES_MAXIT = 4,     /* GMRES reached its restart cap without converging */
  IMEX_NEWTON_MAXIT = 5,    /* nested Newton reached Pnewton_max */
  IMEX_NONFINITE = 6,       /* a NaN or Inf appeared in a solve */
  IMEX_POSITIVITY = 7,      /* p < theta * p_floor after a floored pressure solve */
  IMEX_ERR_SYNC = 8,        /* a device-wide barrier timed out (kernel returned early) */
  IMEX_ERR_EOS = 9          /* a per-cell EOS Newton iteration hit its cap */
} imex_status;

/* Enumerations: names and ordinals of the reference include/config.hpp:27-41,118. */
typedef enum { IMEX_EnergyFormula = 0, IMEX_PressureFormula = 1 } imex_formula;
typedef enum { IMEX_StaggerCT = 0, IMEX_UnStaggerCT = 1, IMEX_PotentialA = 2, IMEX_NoDivFree = 3 } imex_magfield;
typedef enum { IMEX_NoRecon = 0, IMEX_Minmod = 1, IMEX_VanLeer = 2, IMEX_ENO3 = 3, IMEX_WENO5 = 4 } imex_reconstruction;
typedef enum { IMEX_PrimState = 0, IMEX_ConsState = 1 } imex_recon_state;
typedef enum { IMEX_Fullydt = 0, IMEX_Alfvendt = 1, IMEX_IMEXdt = 2 } imex_dt_calculation;
typedef enum { IMEX_x_Transmissive = 0, IMEX_x_Reflective = 1, IMEX_x_Periodic = 2, IMEX_x_Dirichlet = 3 } imex_x_bc;
typedef enum {
  IMEX_y_Transmissive = 0, IMEX_y_Reflective = 1, IMEX_y_Periodic = 2, IMEX_y_Dirichlet = 3, IMEX_y_JetInflow = 4
} imex_y_bc;
typedef enum { IMEX_MaterialSpeedp = 0, IMEX_AlfvenSpeedp = 1, IMEX_Noaddvisp = 2 } imex_add_pvisc;
typedef enum { IMEX_ConservationofU = 0, IMEX_DefinitionofU = 1 } imex_energy_update;
typedef enum { IMEX_Local_Diss = 0, IMEX_Global_Diss = 1 } imex_flux_diss;
typedef enum { IMEX_no_correction = 0, IMEX_once_correction = 1, IMEX_all_correction = 2 } imex_solve_pressure;
typedef enum { IMEX_IDEAL_GAS = 0, IMEX_REDLICH_KWONG = 1 } imex_eos_type;

/* Arithmetic of the implicit solves. */
typedef enum {
  IMEX_PRECISION_FP64 = 0,  /* everything in FP64 (the plain form) */
  IMEX_PRECISION_MIXED = 1  /* FP32 operator + Krylov vectors inside FP64 iterative refinement: every
                               GMRES solve refines in FP64 around FP32 inner cycles; the nested
                               Newton keeps its FP64 residual and convergence test and solves its
                               Jacobian systems in FP32 */
} imex_precision;
/* Operation order of the explicit stencil kernels (reconstruction and the Rusanov face
 * fluxes), imex_config.arith.  The exact order is the reference's, operand for operand,
 * without fused multiply-adds, so those sub-steps match the reference bit for bit.  The
 * fast order hoists the divisions that the reference repeats (WENO5 forms its three
 * nonlinear weights with one division instead of six; the fluxes take 1/rho once) and
 * fuses multiply-adds; a sub-step then differs from the reference by a few units in the
 * last place.  The implicit solves are not affected. */
typedef enum {
  IMEX_ARITH_EXACT = 0,
  IMEX_ARITH_FAST = 1
} imex_arith;
/* Solves of the mixed form (imex_config.mixed_solves).  The pressure solves (the nested
 * Newton's Jacobian systems, or the single linear GMRES without the floor) gain from FP32:
 * the Newton iteration is their FP64 refinement.  The B-form magnetic system (StaggerCT,
 * UnStaggerCT, NoDivFree) gains where it needs many Krylov steps, as on the low-beta random
 * field; the A-form (PotentialA) system converges in a few FP64 steps on the smooth fields
 * of a stage, where FP32 rounding noise costs more refinement sweeps than it saves.  The
 * default is IMEX_MIXED_PRESSURE | IMEX_MIXED_MAGNETIC_B; IMEX_MIXED_MAGNETIC takes both
 * magnetic forms. */
enum { IMEX_MIXED_PRESSURE = 1, IMEX_MIXED_MAGNETIC = 2, IMEX_MIXED_MAGNETIC_B = 4 };

/* Run-time form of the reference's compile-time configuration
 * (include/config.hpp:43-125 and the per-test settings of main.cpp:9-224).
 * Field names follow the reference globals. */
typedef struct imex_config {
  int caltimestep;     /* imex_dt_calculation      (config.hpp:43) */
  int formula;         /* imex_formula             (config.hpp:44) */
  int magfield;        /* imex_magfield            (config.hpp:45) */
  int add_pvisc;       /* imex_add_pvisc           (config.hpp:46) */
  int flux_diss;       /* imex_flux_diss           (config.hpp:47) */
  int GLF;             /* 1: global Lax-Friedrichs dissipation; 0: local, per face (config.hpp:48) */
  int add_bvisc;       /* A-form numerical viscosity (config.hpp:49) */
  int U_update;        /* imex_energy_update       (config.hpp:50) */
  int vortex_test;     /* nonzero reproduces `test == testMHD_vortex` (Minmod y-slope special case) */
  int RKs;             /* IMEX-RK stages: 1, 2 or 3 (config.hpp:56) */
  double CFL;          /* (config.hpp:57) */
  int recon;           /* imex_reconstruction      (config.hpp:60) */
  int reconstate;      /* imex_recon_state         (config.hpp:61) */
  int x_bc, y_bc;      /* imex_x_bc / imex_y_bc (config.hpp:63-64): Periodic or Transmissive, per
                          direction; the other kinds return IMEX_ERR_UNSUPPORTED */
  int PressureSolver;  /* imex_solve_pressure      (config.hpp:65) */
  int Energy_Modify;   /* (config.hpp:69) */
  double GMREStol;     /* (config.hpp:71) */
  double shock_kappa1; /* (config.hpp:77) */
  int floor_on;        /* pressure-positivity nested Newton (config.hpp:100) */
  double p_floor;      /* (config.hpp:101) */
  double Mbig_fac;     /* (config.hpp:102) */
  double theta;        /* (config.hpp:103) */
  int Pnewton_max;     /* (config.hpp:106) */
  double Pnewton_tol;  /* (config.hpp:107) */
  int eos_type;        /* imex_eos_type            (config.hpp:119) */
  double gamma_plasma; /* (config.hpp:122) */
  double m_alfa, m_b, m_R, m_cv; /* Redlich-Kwong constants (config.hpp:125) */
  double x_0, x_1, y_0, y_1;     /* domain (main.cpp:9-224) */
  double time_stop;    /* end time; dt is clipped to reach it (main.cpp:341) */
  double fixed_dt;     /* g_fixed_dt: > 0 forces dt (config.hpp:249) */
  /* additions of this implementation */
  int gmres_restart;      /* Krylov vectors per cycle; the reference hard-codes 25 (implicit_operators.cpp:801) */
  int gmres_max_restarts; /* restart cap; 0 = the vector dimension, as the reference (implicit_operators.cpp:802) */
  int precision;          /* imex_precision */
  double mixed_inner_tol; /* relative tolerance of each FP32 inner solve in mixed mode */
  int mixed_max_refine;   /* cap on FP64 refinement sweeps in mixed mode */
  int mixed_solves;       /* which solves take the mixed form: IMEX_MIXED_* flags */
  double mixed_outer_tol; /* relative residual at which the FP64 refinement of a mixed GMRES solve stops
                             (plus the same value absolute, as GMREStol); the plain form's GMREStol when
                             0.  The default, 1e-10, spends part of the mixed form's 1e-8 error budget. */
  int arith;              /* imex_arith of the explicit stencil kernels; default IMEX_ARITH_FAST */
} imex_config;

/* Scalars that the reference keeps in hidden globals and that one stage consumes
 * (dt, adt, B_max_x/y, vx_max/vy_max, a_max; timestep.cpp:5-67,254-273). */
typedef struct imex_step_scalars {
  double dt, adt, B_max_x, B_max_y, vx_max, vy_max, v_max, a_max, ch, cA_x, cA_y, t;
  int timestep;
} imex_step_scalars;

/* Counters of the implicit solves, accumulated since the last imex_reset_stats. */
typedef struct imex_solve_stats {
  int gmres_solves;      /* GMRES calls */
  int gmres_iters;       /* Arnoldi steps (operator applications inside cycles) */
  int gmres_restarts;    /* restart cycles */
  int newton_iters;      /* nested-Newton Jacobian solves */
  int max_floored;       /* largest number of cells below p_floor after a Newton solve */
  int refine_sweeps;     /* FP64 refinement sweeps (mixed precision) */
  double last_residual;  /* residual estimate at exit of the last GMRES solve */
  double min_p;          /* smallest pressure after a floored solve */
  int status;            /* worst imex_status seen */
} imex_solve_stats;

typedef struct imex_ctx imex_ctx;

/* Context and configuration ------------------------------------------------ */
void imex_config_default(imex_config* cfg); /* the reference defaults, config.hpp:43-125 */
imex_status imex_create(const imex_config* cfg, int nx, int ny, imex_ctx** out);
imex_status imex_destroy(imex_ctx* ctx);
imex_status imex_set_stream(imex_ctx* ctx, void* cuda_stream); /* cudaStream_t; NULL = own stream */
imex_status imex_synchronize(imex_ctx* ctx);
const char* imex_status_string(imex_status s);
const char* imex_last_error(const imex_ctx* ctx);
imex_status imex_get_config(const imex_ctx* ctx, imex_config* cfg);

/* State I/O ---------------------------------------------------------------- */
/* Initial data as primitive planes + faces + vector potential; converts to conserved
 * like main.cpp:240-244 (u_initialization, upri2ucon, A_initial). */
imex_status imex_upload_prim(imex_ctx* ctx, const double* prim8, const double* bx, const double* by,
                             const double* A3);
/* Same as imex_upload_prim but keeps the simulation time, step counter and dt history,
 * so a driver can hand the solver a state it holds in host memory at every step. */
imex_status imex_upload_state(imex_ctx* ctx, const double* prim8, const double* bx, const double* by,
                              const double* A3);
/* Current state; any pointer may be NULL. */
imex_status imex_download_state(imex_ctx* ctx, double* cons8, double* prim8, double* bx, double* by, double* A3);
/* Boundary normal faces of a transmissive direction: Bx on x = x_0 (ny values, one per row)
 * and By on y = y_0 (nx values, one per column).  The reference carries them as the faces
 * at ghost index ghost_cells - 1 of Bx_p0 / By_0p, which bound_cond_staggered preserves and
 * Staggered_CT_Consistent evolves (constrained_transport.cpp:5-30, ct_flux.cpp:176-189);
 * the bx / by planes above hold the faces at i + 1/2 and j + 1/2 of the interior cells only.
 * imex_upload_prim sets them to the first interior face of their row / column (Bx(1/2, j),
 * By(i, 1/2)); set them after it to the initial condition's own values.  A NULL pointer or a
 * periodic direction leaves that line alone.  Reading a periodic direction returns the
 * faces it identifies with x_0 / y_0, those at x_1 / y_1.  Host or device pointers. */
imex_status imex_set_boundary_faces(imex_ctx* ctx, const double* bx_x0, const double* by_y0);
imex_status imex_get_boundary_faces(imex_ctx* ctx, double* bx_x0, double* by_y0);

/* Time stepping ------------------------------------------------------------ */
/* One full time step of main.cpp:335-561: global wave-speed maxima, dt, every stage. */
imex_status imex_step(imex_ctx* ctx, double* dt_out);
/* Step prologue alone (main.cpp:335-366): scalars, dt, u^n snapshot. */
imex_status imex_begin_step(imex_ctx* ctx);
/* One IMEX stage (main.cpp:367-559 body for stage rks). */
imex_status imex_stage(imex_ctx* ctx, int rks);
/* Step epilogue (main.cpp:561): primitive state of the new step. */
imex_status imex_end_step(imex_ctx* ctx);
imex_status imex_set_step_scalars(imex_ctx* ctx, const imex_step_scalars* s);
imex_status imex_get_step_scalars(imex_ctx* ctx, imex_step_scalars* s);

/* Sub-steps of one stage, in the order of main.cpp:368-555.  Each reads and writes
 * the context's stage buffers (imex_buffer) exactly as the reference function
 * reads and writes its arguments. */
imex_status imex_stage_combine(imex_ctx* ctx, int rks);                       /* main.cpp:368-414 */
imex_status imex_TVDReconstruction(imex_ctx* ctx);                            /* reconstruction.cpp:5 (Qe -> w) */
imex_status imex_RusanovC_Update(imex_ctx* ctx, double h, int rks);           /* flux.cpp:409 */
imex_status imex_MagSubsystem_UpdateB(imex_ctx* ctx, double h, int rks);      /* imex_subsystems.cpp:537 */
imex_status imex_MagSubsystem_UpdateA(imex_ctx* ctx, double h, int rks);      /* imex_subsystems.cpp:5 */
imex_status imex_Pressure_flux_Update(imex_ctx* ctx, double h, int rks);      /* flux.cpp:290 + main.cpp:447-467 */
imex_status imex_PreSubsystem_Pressure(imex_ctx* ctx, double h, int rks);     /* imex_subsystems.cpp:76 */
imex_status imex_Energy_flux_Update(imex_ctx* ctx, double h, int rks);        /* flux.cpp:163 + main.cpp:447-467 */
imex_status imex_PreSubsystem_Energy(imex_ctx* ctx, double h, int rks);       /* imex_subsystems.cpp:415 */
imex_status imex_Staggered_CT_Consistent(imex_ctx* ctx, double h, int rks);   /* ct_flux.cpp:150 */
imex_status imex_Unstaggered_CT_Consistent(imex_ctx* ctx, double h, int rks); /* constrained_transport.cpp:500 */
imex_status imex_Staggered_CT(imex_ctx* ctx, double h, int rks);             /* constrained_transport.cpp:66 */
imex_status imex_Unstaggered_CT(imex_ctx* ctx, double h, int rks);           /* constrained_transport.cpp:436 */
imex_status imex_stage_derivative(imex_ctx* ctx, int rks);                    /* main.cpp:537-555 */

/* Stage buffers, for drivers and tests that run sub-steps individually. */
typedef enum imex_buffer {
  IMEX_BUF_CONS = 0,  /* u_con, 8 planes */
  IMEX_BUF_PRIM = 1,  /* u_pri, 8 planes */
  IMEX_BUF_CONS_N = 2,/* u_con_n (state at the start of the step), 8 planes */
  IMEX_BUF_QE = 3,    /* explicit stage state Qe, 8 planes */
  IMEX_BUF_QS = 4,    /* implicit stage state Qs, 8 planes */
  IMEX_BUF_BX = 5,    /* Bx_p0 faces */
  IMEX_BUF_BY = 6,    /* By_0p faces */
  IMEX_BUF_BX_QS = 7, /* Bx_p0_Qs */
  IMEX_BUF_BY_QS = 8, /* By_0p_Qs */
  IMEX_BUF_A = 9,     /* A, 3 planes */
  IMEX_BUF_A_S = 10,  /* A_s, 3 planes */
  IMEX_BUF_FLUX_X = 11, /* gFluxBy_p0 */
  IMEX_BUF_FLUX_Y = 12, /* gFluxBx_0p */
  IMEX_BUF_W = 13,    /* reconstruction w_xL, w_xR, w_yL, w_yR: 32 planes */
  IMEX_BUF_HS = 14,   /* Hs[index], 8 planes */
  IMEX_BUF_HSA = 15,  /* HsA[index], 3 planes */
  IMEX_BUF_HSB = 16,  /* HsB[index], 2 planes */
  IMEX_BUF_SHOCK = 17, /* shock detector eta of the last pressure solve, 1 plane */
  IMEX_BUF_BX_X0 = 18,    /* transmissive x: Bx_p0 on x = x_0, ny values */
  IMEX_BUF_BY_Y0 = 19,    /* transmissive y: By_0p on y = y_0, nx values */
  IMEX_BUF_BX_QS_X0 = 20, /* the same lines of Bx_p0_Qs / By_0p_Qs */
  IMEX_BUF_BY_QS_Y0 = 21
} imex_buffer;
imex_status imex_buffer_count(const imex_ctx* ctx, int buffer, size_t* ndoubles);
imex_status imex_set_buffer(imex_ctx* ctx, int buffer, int index, const double* src);
imex_status imex_get_buffer(imex_ctx* ctx, int buffer, int index, double* dst);

/* Operators, GMRES and the nested Newton --------------------------------- */
typedef enum imex_op {
  IMEX_OP_PRESSURE_L = 0, /* Pressure_Subsystem_AX, g_AX_jacobian = false (implicit_operators.cpp:505) */
  IMEX_OP_PRESSURE_J = 1, /* Pressure_Subsystem_AX, g_AX_jacobian = true */
  IMEX_OP_MAGNETIC_B = 2, /* Magnetic_Subsystem_AX (implicit_operators.cpp:141) */
  IMEX_OP_MAGNETIC_A = 3, /* Magnetic_Subsystem_potential_AX (implicit_operators.cpp:355) */
  IMEX_OP_ENERGY = 4      /* Energy_Subsystem_AX (implicit_operators.cpp:741) */
} imex_op;
/* Freeze the coefficients of `op` from the current CONS (rho), QE and QS buffers,
 * exactly what the reference operator reads on each application. */
imex_status imex_prepare_operator(imex_ctx* ctx, int op, double h);
/* Newton state for IMEX_OP_PRESSURE_J: p_freeze (one plane) and Mbig (config.hpp:104,108). */
imex_status imex_set_newton_state(imex_ctx* ctx, const double* p_freeze, double mbig);
/* Ax = op(x), no preconditioner (the reference X_Subsystem_AX functions). */
imex_status imex_apply_operator(imex_ctx* ctx, int op, const double* x, double* Ax);
/* GMRES_Solver (implicit_operators.cpp:793): x in/out, b in.  The pressure operators use
 * the reference's Jacobi preconditioner precP (implicit_operators.cpp:650), the magnetic
 * ones none, as in the reference call sites. */
imex_status imex_gmres(imex_ctx* ctx, int op, double* x, const double* b, imex_solve_stats* stats);
/* imex_gmres without any allocation.  This entry point has no counterpart in the
 * reference (whose GMRES_Solver allocates its Krylov and work vectors on every
 * call, implicit_operators.cpp:808-810); it is an addition of this implementation.
 *
 * imex_gmres takes its temporaries for host x/b from cudaMallocAsync.  Callers that
 * cannot enter the device allocator during a solve use this one instead: a host
 * whose own allocator has reserved the device's free memory (a cudaMalloc would
 * fail or force that allocator to release memory), and a per-step loop with a hard
 * latency budget, where an allocation may block on the pool.  Here the Krylov
 * basis, the AV ring, the per-CTA partial sums, the barrier state and the staged
 * host vectors all live in one fixed device array of IMEX_NOALLOC_SCRATCH_BYTES
 * (16 MiB) per device; no cudaMalloc, cudaFree or other allocating call is made.
 * Same kernel, same arithmetic and same results as imex_gmres in the FP64 form
 * (it always solves in FP64, whatever the context's precision).
 *
 * Limit: the solve needs about (gmres_restart + 3) x unknowns x 8 bytes, plus
 * 2 x unknowns x 8 bytes when x or b are host pointers.  For restart 25 that is
 * up to ~73,000 pressure unknowns (256 x 256 cells) or ~24,000 cells for the
 * magnetic systems (3 unknowns per cell).  Larger solves are rejected with
 * IMEX_ERR_INVALID before any work, and imex_last_error names the bytes needed.
 *
 * The first call on a device resolves the array's address (cudaGetSymbolAddress,
 * with that device current).  Every call synchronizes the context's stream and then
 * reads the solve's status, so it must not be made while that stream is being
 * captured into a CUDA graph.  The barrier state in the array is cleared by every call.  The array is shared by
 * every context and stream on a device, so calls that overlap in time on one
 * device race: serialise them. */
#define IMEX_NOALLOC_SCRATCH_BYTES ((size_t)16 << 20)
imex_status imex_gmres_noalloc(imex_ctx* ctx, int op, double* x, const double* b, imex_solve_stats* stats);
/* Pressure_NestedNewton (implicit_operators.cpp:625): p in/out, b in. */
imex_status imex_pressure_nested_newton(imex_ctx* ctx, double* p, const double* b, imex_solve_stats* stats);
/* ShockDetector (flux.cpp:5) of 8 conserved planes into one plane. */
imex_status imex_shock_detector(imex_ctx* ctx, const double* Q8, double* eta);

/* Ensembles ------------------------------------------------------------------
 * Many independent runs of the same configuration on uneven grids, advanced together
 * (no counterpart in the reference, which runs one grid per process).  Member m is an
 * ordinary context of nx[m] x ny[m] cells: its data go in and out through the usual
 * entry points (imex_upload_prim, imex_download_state, imex_divergence, ...) on the
 * handle from imex_batch_member, and it keeps its own dt, time and statistics.
 * imex_batch_step advances every member by `steps` time steps: each explicit sub-step
 * is one launch for all members (or, with imex_batch_configure(b, streams > 0, ...), the
 * members launch their own kernels on a pool of streams), and each implicit solve of a
 * stage is one cooperative launch for all members, in which each member owns a range of
 * CTAs.  The step is captured once into a CUDA graph and replayed.  Members must share the RK
 * order and the magnetic form; imex_batch_step synchronises and returns the worst
 * member status (imex_batch_last_error names the member). */
/* ---- output formats and run diagnostics (main.cpp:560-721, output.cpp)
 * The per-step quantities the reference prints and records after every step. */
typedef struct imex_diagnostics_t {
  int timestep;
  double t, dt;
  double div_error;  /* cal_divergence_error (imex_subsystems.cpp:630): face FV L2 for StaggerCT, else cell L2 */
  double B_inf;      /* max |central div of cell B| (main.cpp:578-589) */
  double dt_comp;    /* imex_dt / fully_dt (timestep.cpp:56-57) */
  double emin, emin_x, emin_y;  /* min internal energy and its cell centre (main.cpp:562-573) */
  double mass, intE;            /* integrals of rho and of the internal energy over the domain */
  double magE_max;              /* max |B|^2 / 2 */
} imex_diagnostics_t;
imex_status imex_diagnostics(imex_ctx* ctx, imex_diagnostics_t* d);
/* Diagnose_CT_EMF (constrained_transport.cpp:166-222), which the reference's driver prints
 * after every step (main.cpp:594): the corner EMF of the current state split into its parts
 * from the central face average, the Rusanov dissipation and the cell EMF Ez~, and their sum.
 * out[4 c + q] for c = central, rusanov, tilde, total and q = L2 of Ez, max |Ez|, L2 of the
 * face injection rate |dB/dt|, its max.  Overwrites the reconstruction buffer (IMEX_BUF_W)
 * and the stage work planes, which only the inside of a stage reads. */
imex_status imex_ct_emf_diagnostics(imex_ctx* ctx, double* out16);
/* Legacy-VTK rectilinear grid of the current state: the reference's 13 cell fields (rho,
 * mom_X/Y/Z, U, B_X/Y/Z, velX/Y/Z, p, B), node coordinates on the nx + 1 / ny + 1 cell faces,
 * interior cells only, 17 significant digits. */
imex_status imex_write_vtk(imex_ctx* ctx, const char* path, int cycle);
/* The final-state field files RK_rho/vx/vy/E/p/Bx/By/Bz/v_mag.dat (and RK_T.dat for the
 * Redlich-Kwong EOS) into `dir`: "x y value" per cell, x outer, full precision. */
imex_status imex_write_fields_dat(imex_ctx* ctx, const char* dir);
/* Binary state (primitive planes, faces, A, t, step counter, previous dt; a transmissive run
 * also its boundary normal faces, file version 2): a run loaded from it continues bit for bit. */
imex_status imex_save_state_file(imex_ctx* ctx, const char* path);
imex_status imex_load_state_file(imex_ctx* ctx, const char* path);
/* The writers on host arrays (no GPU needed); "timestep value" lines for the histories. */
int imex_vtk_write_host(const char* path, int nx, int ny, double x0, double y0, double dx, double dy, double t,
                        int cycle, const double* cons8, const double* prim8);
int imex_dat_write_host(const char* path, int nx, int ny, double x0, double y0, double dx, double dy,
                        const double* plane);
int imex_history_write_host(const char* path, int n, const int* steps, const double* values);

/* ---- discrete adjoint
 * Gradients of the final state of an nsteps run with respect to the initial fields, by the
 * hand-written discrete adjoint of the step: every sub-step of main.cpp:335-561 in reverse,
 * each implicit solve as a transposed matrix-free GMRES solve on the assembled transposed
 * stencil, the nested Newton differentiated at its converged pressure through its active set
 * (with the Cor.1 slope Mbig), the GLF maxima through the cells attaining them.  Checkpoints
 * every `checkpoint_every` steps; each segment and each step are recomputed from them.
 * Supported: PressureFormula, StaggerCT, ConsState or PrimState, ideal gas, GLF, any
 * pressure viscosity, fixed_dt > 0, FP64, DefinitionofU or ConservationofU, Energy_Modify
 * on or off, periodic boundaries (else IMEX_ERR_UNSUPPORTED).
 * The run starts from the context's current state and leaves it at the final state. */
typedef struct imex_adjoint_opts {
  int nsteps;            /* steps of the forward run (>= 1) */
  int checkpoint_every;  /* steps between checkpoints (>= 1) */
  double gmres_tol;      /* relative tolerance of the transposed solves (<= 0: 1e-13) */
} imex_adjoint_opts;
/* J = 1/2 |rho(T) - rho_target|^2 + 1/2 |B(T) - B_target|^2 (cell values, B_target three
 * planes) and its gradient with respect to the initial primitive planes (8) and face fields.
 * Host or device pointers; J, g_prim, g_bx, g_by may be NULL. */
imex_status imex_adjoint_run(imex_ctx* ctx, const imex_adjoint_opts* opts, const double* rho_target,
                             const double* B_target, double* J, double* g_prim, double* g_bx, double* g_by);
/* The vector-Jacobian product for a given cotangent of the final conserved planes (8) and
 * faces (lam_bx, lam_by may be NULL). */
imex_status imex_adjoint_vjp(imex_ctx* ctx, const imex_adjoint_opts* opts, const double* lam_cons,
                             const double* lam_bx, const double* lam_by, double* g_prim, double* g_bx, double* g_by);

typedef struct imex_batch imex_batch;
typedef struct imex_batch_tuning {
  int streams;          /* streams of the explicit sub-steps (0: one batched launch per sub-step) */
  int gmres_restart;    /* Krylov vectors per cycle of every member */
  double ms_per_step;   /* device time of one ensemble step at that choice */
  int mixed_solves;     /* IMEX_MIXED_* flags of every member (mixed precision only) */
  int solve_tile_x, solve_tile_y;  /* cells per tile of the batched B-form magnetic solve */
} imex_batch_tuning;
imex_status imex_batch_create(const imex_config* cfg, int members, const int* nx, const int* ny, imex_batch** out);
imex_status imex_batch_destroy(imex_batch* b);
imex_status imex_batch_member(imex_batch* b, int m, imex_ctx** ctx);
/* how the explicit sub-steps run, and graph capture (default on).  streams = 0 (the
 * default): each explicit sub-step is one launch for all members, whose grids are laid end
 * to end (the step is planned once by recording every member's launches); streams > 0:
 * every member launches its own kernels, the members spread over that many streams. */
imex_status imex_batch_configure(imex_batch* b, int streams, int use_graph);
/* advance every member `steps` steps; *device_ms (optional) = device time of those steps */
imex_status imex_batch_step(imex_batch* b, int steps, double* device_ms);
/* launches of one ensemble step in the batched mode: the explicit sub-steps, and the
 * batched solves (a barrier reset and a cooperative launch per chunk); -1 in the streams
 * mode.  The second pointer may be null. */
imex_status imex_batch_explicit_launches(imex_batch* b, int* launches_per_step, int* solve_launches_per_step);
/* tile shape of the batched B-form magnetic solve in the fast arithmetic: 0 = 32 x 16 cells
 * (the default, and the shape of every single-context solve), 1 = 64 x 8, 2 = 32 x 8 */
imex_status imex_batch_set_solve_tile(imex_batch* b, int tile);
/* time `trial_steps` ensemble steps per candidate, one choice at a time from the best so
 * far: the explicit mode (batched launches, or 4 / 8 / 16 streams), the B-form solve's tile
 * shape (B form, fast arithmetic), the restart length (15 or the configured one) and, in
 * mixed precision, the configured mixed_solves or the same with the magnetic systems' FP32
 * form toggled; restore every member's state after each trial and keep the fastest */
imex_status imex_batch_autotune(imex_batch* b, int trial_steps, imex_batch_tuning* out);
/* streams in use, whether the step runs as a captured graph, batched solve launches per step */
imex_status imex_batch_info(imex_batch* b, int* streams, int* graph_used, int* solve_launches_per_step);
const char* imex_batch_last_error(const imex_batch* b);

/* Statistics and diagnostics ---------------------------------------------- */
imex_status imex_get_stats(imex_ctx* ctx, imex_solve_stats* stats);
imex_status imex_reset_stats(imex_ctx* ctx);
/* Divergence of B (imex_subsystems.cpp:630): face finite-volume L2 of the staggered
 * field; L2 of the periodic central difference of cell B; the reference's own
 * cell metric (one-sided at the domain edge); max |central div| of cell B. */
imex_status imex_divergence(imex_ctx* ctx, double* face_l2, double* cell_wrapped_l2, double* cell_ref_l2,
                            double* cell_inf);
/* Failure detection ---------------------------------------------------------
 * Every device-wide wait inside the persistent solver kernels is bounded: after
 * `seconds` (default 2 s) the waiting CTAs give up, the kernel returns and the
 * call reports IMEX_ERR_SYNC; the context stays usable. */
imex_status imex_set_barrier_timeout(imex_ctx* ctx, double seconds);
/* Runs `iterations` device-wide barriers with the solver's CTA count and reports the
 * mean cost per barrier.  `phantom_blocks` > 0 makes the barrier wait for CTAs that
 * were never launched, so the bounded wait must run out after `timeout_s` and the
 * call must return IMEX_ERR_SYNC (a self-test of the failure path). */
imex_status imex_selftest_barrier(imex_ctx* ctx, int iterations, int phantom_blocks, double timeout_s,
                                  double* us_per_barrier);
/* FP64 throughput of the context's device, measured (no counterpart in the reference):
 * fused multiply-adds per second and IEEE double divisions per second, each from a
 * kernel of independent dependency chains over every SM with no memory traffic.  These
 * are the denominators against which a stencil kernel is called FP64 bound. */
imex_status imex_selftest_fp64(imex_ctx* ctx, double* dfma_per_s, double* ddiv_per_s);
/* Minimum pressure of the current primitive state. */
imex_status imex_min_pressure(imex_ctx* ctx, double* pmin);

/* Live kernel profile -------------------------------------------------------
 * With profiling on, every kernel launch family is bracketed by CUDA events on the
 * context's stream and its algorithmic HBM bytes (compulsory traffic: each input
 * read once, each output written once) are accumulated; the persistent solver
 * kernels count their own phases on the device. */
typedef struct imex_kernel_profile {
  char name[32];
  long long launches;
  double total_ms;     /* sum of event-timed durations */
  double alg_bytes;    /* algorithmic bytes over all launches */
} imex_kernel_profile;
imex_status imex_profile_enable(imex_ctx* ctx, int on); /* also clears the counters */
/* Fills up to `max` entries (families with at least one launch); *count = entries written. */
imex_status imex_profile_read(imex_ctx* ctx, imex_kernel_profile* out, int max, int* count);
/* Number of CUDA kernels this context has launched since it was created. */
imex_status imex_kernel_launch_count(const imex_ctx* ctx, long long* count);

#ifdef __cplusplus
}
#endif
#endif /* IMEX_B200_H */
