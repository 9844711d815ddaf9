// Reference harness: drives the reference solver's OWN code as a library.
//
// Test infrastructure only (the oracle).  Nothing in the product links this.
//
// Build (oracle/Makefile): the reference sources are copied to a scratch
// directory outside this repository, the three grid-size constants of
// include/config.hpp are made run-time settable (`const int nxCells` ->
// `inline int nxCells`, same for nyCells and RKs), and two fragments of
// src/main.cpp are cut out verbatim into include files:
//   ref_tableau.inc   = main.cpp:269-319  (Butcher tableaux)
//   ref_step_body.inc = main.cpp:335-561  (one time step: BCs, calch/caldt,
//                        eigenvalues, con<->prim, the IMEX stage loop
//                        main.cpp:367-559, final con->prim)
// and the same time step once more in three pieces, so that a caller can advance
// the reference one IMEX stage at a time (ref_stage):
//   ref_step_pre.inc   = main.cpp:335-366  (the part before the stage loop; its
//                        local `Grid A_n_snapshot` becomes a reference to a grid
//                        held here, because it must outlive the call)
//   ref_stage_body.inc = main.cpp:368-558  (the body of the stage loop)
//   ref_step_post.inc  = main.cpp:561      (final con->prim)
// Every other reference .cpp except main.cpp is compiled unchanged and linked
// in.  This file supplies what main() would: allocation, initial-data
// injection, and read-back.  Sub-step calls inside the stage loop are wrapped
// by macros that snapshot the state after each sub-step, so tests can compare
// a GPU sub-step with the reference on identical inputs.
//
// All arrays exchanged through the C interface are interior-only SoA planes
// of nx*ny doubles, index i + nx*j (x fastest), the same order the reference
// uses for its GMRES vectors (M_P / M_B, implicit_operators.cpp:5-139).
// Face fields use the same shape: plane(i,j) holds Bx_p0 at (i+1/2, j) and
// By_0p at (i, j+1/2).

#include "declarations.hpp"

#include <cstdio>
#include <cstring>
#include <vector>

#include <fcntl.h>
#include <unistd.h>

namespace {

struct Snap {
  bool valid = false;
  std::vector<double> u_con, Qe, Qs, bx, by, bxQs, byQs, A, A_s, Fx, Fy;
};

enum { SUB_COMBINE = 0, SUB_CONVECTIVE, SUB_MAGNETIC, SUB_PFLUX, SUB_PRESSURE, SUB_CT, NSUB };
const int MAXRK = 3;

struct State {
  bool ready = false;
  Grid *u_pri = nullptr, *u_con = nullptr, *u_con_n = nullptr, *Qe = nullptr, *Qe_pri = nullptr,
       *Qs = nullptr, *w_xL = nullptr, *w_xR = nullptr, *w_yL = nullptr, *w_yR = nullptr, *A = nullptr,
       *A_n_snapshot = nullptr;
  Tensor *HsA = nullptr, *HsB = nullptr, *Hs = nullptr;
  Array *Bx_p0 = nullptr, *By_0p = nullptr, *Bx_p0_n = nullptr, *By_0p_n = nullptr, *Bx = nullptr,
        *By = nullptr, *Bz = nullptr, *Bx_p0_Qe = nullptr, *By_0p_Qe = nullptr, *Bx_p0_Qs = nullptr,
        *By_0p_Qs = nullptr, *Ae = nullptr, *Ai = nullptr;
  bool snap_on = false;
  int next_stage = 0;  // ref_stage: the stage the next call runs (0 = a new time step)
  Snap snaps[MAXRK][NSUB];
};
State S;

template <class T> void del(T*& p) {
  delete p;
  p = nullptr;
}

void free_all() {
  del(S.u_pri); del(S.u_con); del(S.u_con_n); del(S.Qe); del(S.Qe_pri); del(S.Qs);
  del(S.w_xL); del(S.w_xR); del(S.w_yL); del(S.w_yR); del(S.A); del(S.A_n_snapshot);
  del(S.HsA); del(S.HsB); del(S.Hs);
  del(S.Bx_p0); del(S.By_0p); del(S.Bx_p0_n); del(S.By_0p_n); del(S.Bx); del(S.By); del(S.Bz);
  del(S.Bx_p0_Qe); del(S.By_0p_Qe); del(S.Bx_p0_Qs); del(S.By_0p_Qs); del(S.Ae); del(S.Ai);
  del(gFluxBy_p0); del(gFluxBx_0p);
  S.ready = false;
}

inline int PX() { return nxCells + 2 * ghost_cells; }
inline int PY() { return nyCells + 2 * ghost_cells; }
inline size_t gsize() { return (size_t)PX() * PY() * NUM_VARS; }
inline size_t asize() { return (size_t)PX() * PY(); }

void grid_from_planes(Grid& g, const double* planes, int nvar) {
  const int nx = nxCells, ny = nyCells;
  for (int k = 0; k < nvar; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        g(i + ghost_cells, j + ghost_cells, k) = planes[(size_t)k * nx * ny + i + (size_t)nx * j];
}
void grid_to_planes(const Grid& g, double* planes, int nvar) {
  const int nx = nxCells, ny = nyCells;
  for (int k = 0; k < nvar; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        planes[(size_t)k * nx * ny + i + (size_t)nx * j] = g(i + ghost_cells, j + ghost_cells, k);
}
void array_from_plane(Array& a, const double* p) {
  for (int j = 0; j < nyCells; ++j)
    for (int i = 0; i < nxCells; ++i) a(i + ghost_cells, j + ghost_cells) = p[i + (size_t)nxCells * j];
}
void array_to_plane(const Array& a, double* p) {
  for (int j = 0; j < nyCells; ++j)
    for (int i = 0; i < nxCells; ++i) p[i + (size_t)nxCells * j] = a(i + ghost_cells, j + ghost_cells);
}
void zero_grid(Grid& g) { std::memset(g.data, 0, gsize() * sizeof(double)); }
void zero_array(Array& a) { std::memset(a.data, 0, asize() * sizeof(double)); }

void save_grid(std::vector<double>& v, const Grid& g) { v.assign(g.data, g.data + gsize()); }
void save_array(std::vector<double>& v, const Array& a) { v.assign(a.data, a.data + asize()); }

void snapshot(int sub, int rks, Grid& u_con, Grid& Qe, Grid& Qs, Array& bx, Array& by, Array& bxQs,
              Array& byQs, Grid& A, Grid& A_s) {
  if (!S.snap_on || rks < 0 || rks >= MAXRK) return;
  Snap& s = S.snaps[rks][sub];
  save_grid(s.u_con, u_con);
  save_grid(s.Qe, Qe);
  save_grid(s.Qs, Qs);
  save_array(s.bx, bx);
  save_array(s.by, by);
  save_array(s.bxQs, bxQs);
  save_array(s.byQs, byQs);
  save_grid(s.A, A);
  save_grid(s.A_s, A_s);
  if (gFluxBy_p0) save_array(s.Fx, *gFluxBy_p0);
  if (gFluxBx_0p) save_array(s.Fy, *gFluxBx_0p);
  s.valid = true;
}

void set_tableau() {
  Array& Ae = *S.Ae;
  Array& Ai = *S.Ai;
  std::vector<double> bRK(RKs);
#include "ref_tableau.inc"
  (void)bRK;
}

// The names main() gives the solver state, bound to the grids held here.
#define BIND_STATE \
  Grid& u_pri = *S.u_pri; \
  Grid& u_con = *S.u_con; \
  Grid& u_con_n = *S.u_con_n; \
  Grid& Qe = *S.Qe; \
  Grid& Qe_pri = *S.Qe_pri; \
  Grid& Qs = *S.Qs; \
  Grid& w_xL = *S.w_xL; \
  Grid& w_xR = *S.w_xR; \
  Grid& w_yL = *S.w_yL; \
  Grid& w_yR = *S.w_yR; \
  Grid& A = *S.A; \
  Tensor& HsA = *S.HsA; \
  Tensor& HsB = *S.HsB; \
  Tensor& Hs = *S.Hs; \
  Array& Bx_p0 = *S.Bx_p0; \
  Array& By_0p = *S.By_0p; \
  Array& Bx_p0_n = *S.Bx_p0_n; \
  Array& By_0p_n = *S.By_0p_n; \
  Array& Bx = *S.Bx; \
  Array& By = *S.By; \
  Array& Bz = *S.Bz; \
  Array& Bx_p0_Qe = *S.Bx_p0_Qe; \
  Array& By_0p_Qe = *S.By_0p_Qe; \
  Array& Bx_p0_Qs = *S.Bx_p0_Qs; \
  Array& By_0p_Qs = *S.By_0p_Qs; \
  Array& Ae = *S.Ae; \
  Array& Ai = *S.Ai;

// One time step of the reference driver, main.cpp:335-561, with sub-step hooks.
void run_step_body() {
  BIND_STATE
  bool isFinalTime = false;

#define HOOK_(sub) snapshot(sub, rks, u_con, Qe, Qs, Bx_p0, By_0p, Bx_p0_Qs, By_0p_Qs, A, A_s)
#define TVDReconstruction(...) do { HOOK_(SUB_COMBINE); (TVDReconstruction)(__VA_ARGS__); } while (0)
#define RusanovC_Update(...) do { (RusanovC_Update)(__VA_ARGS__); HOOK_(SUB_CONVECTIVE); } while (0)
#define MagSubsystem_UpdateB(...) do { (MagSubsystem_UpdateB)(__VA_ARGS__); HOOK_(SUB_MAGNETIC); } while (0)
#define MagSubsystem_UpdateA(...) do { (MagSubsystem_UpdateA)(__VA_ARGS__); HOOK_(SUB_MAGNETIC); } while (0)
#define Pressure_flux_Update(...) do { (Pressure_flux_Update)(__VA_ARGS__); HOOK_(SUB_PFLUX); } while (0)
#define Energy_flux_Update(...) do { (Energy_flux_Update)(__VA_ARGS__); HOOK_(SUB_PFLUX); } while (0)
#define PreSubsystem_Pressure(...) do { (PreSubsystem_Pressure)(__VA_ARGS__); HOOK_(SUB_PRESSURE); } while (0)
#define PreSubsystem_Energy(...) do { (PreSubsystem_Energy)(__VA_ARGS__); HOOK_(SUB_PRESSURE); } while (0)
#define Staggered_CT_Consistent(...) do { (Staggered_CT_Consistent)(__VA_ARGS__); HOOK_(SUB_CT); } while (0)
#define Unstaggered_CT_Consistent(...) do { (Unstaggered_CT_Consistent)(__VA_ARGS__); HOOK_(SUB_CT); } while (0)

#include "ref_step_body.inc"

#undef TVDReconstruction
#undef RusanovC_Update
#undef MagSubsystem_UpdateB
#undef MagSubsystem_UpdateA
#undef Pressure_flux_Update
#undef Energy_flux_Update
#undef PreSubsystem_Pressure
#undef PreSubsystem_Energy
#undef Staggered_CT_Consistent
#undef Unstaggered_CT_Consistent
#undef HOOK_
  (void)isFinalTime;
}

// The same time step in three pieces (ref_stage): before the stage loop, one
// pass of the stage loop's body for stage `rks`, and after the loop.  Run in
// order pre, stage 0 .. RKs-1, post, they execute the statements of
// run_step_body() in the same order on the same state (no snapshots).
void run_step_pre() {
  BIND_STATE
  bool isFinalTime = false;
#include "ref_step_pre.inc"
  (void)isFinalTime;
  (void)Qe; (void)Qe_pri; (void)Qs; (void)w_xL; (void)w_xR; (void)w_yL; (void)w_yR;
  (void)HsA; (void)HsB; (void)Hs; (void)Bx; (void)By; (void)Bz; (void)Bx_p0_Qe; (void)By_0p_Qe;
  (void)Bx_p0_Qs; (void)By_0p_Qs; (void)Ae; (void)Ai;
}

void run_stage_body(int rks) {
  BIND_STATE
  Grid& A_n_snapshot = *S.A_n_snapshot;
  bool isFinalTime = false;
#include "ref_stage_body.inc"
  (void)isFinalTime;
  (void)Bx_p0_n; (void)By_0p_n;
}

void run_step_post() {
  Grid& u_pri = *S.u_pri;
  Grid& u_con = *S.u_con;
#include "ref_step_post.inc"
}

}  // namespace

extern "C" {

// Solver settings mirrored from include/config.hpp (names kept).  Enum-valued
// fields take the reference enum ordinals.
struct ref_params {
  int formula, magfield, recon, reconstate, caltimestep, add_pvisc, U_update, PressureSolver, eos_type;
  int GLF, add_bvisc, floor_on, Energy_modify, vortex_test, Pnewton_max;
  double CFL, GMREStol, gamma_plasma, p_floor, Mbig_fac, theta, Pnewton_tol, shock_kappa1;
  double m_alfa, m_b, m_R, m_cv, x0, x1, y0, y1, time_stop, fixed_dt;
};

int ref_setup(int nx, int ny, int rk, const ref_params* p) {
  if (nx < 4 || ny < 4 || rk < 1 || rk > MAXRK) return 1;
  free_all();
  nxCells = nx;
  nyCells = ny;
  RKs = rk;
  nxPoints = nx + 1;
  nyPoints = ny + 1;
  formula = (Formula)p->formula;
  magfield = (MagField)p->magfield;
  recon = (Reconstruction)p->recon;
  reconstate = (ReconState)p->reconstate;
  caltimestep = (dtCalculation)p->caltimestep;
  add_pvisc = (Add_Pvisc)p->add_pvisc;
  U_update = (Energy_Update)p->U_update;
  PressureSolver = (SolvePressure)p->PressureSolver;
  eos_type = (EOSType)p->eos_type;
  GLF = p->GLF != 0;
  add_bvisc = p->add_bvisc != 0;
  floor_on = p->floor_on != 0;
  Energy_Modify = p->Energy_modify != 0;
  test = p->vortex_test ? testMHD_vortex : testOrszag_Tang;
  Pnewton_max = p->Pnewton_max;
  CFL = p->CFL;
  GMREStol = p->GMREStol;
  gamma_plasma = p->gamma_plasma;
  p_floor = p->p_floor;
  Mbig_fac = p->Mbig_fac;
  theta = p->theta;
  Pnewton_tol = p->Pnewton_tol;
  shock_kappa1 = p->shock_kappa1;
  m_alfa = p->m_alfa;
  m_b = p->m_b;
  m_R = p->m_R;
  m_cv = p->m_cv;
  x_0 = p->x0;
  x_1 = p->x1;
  y_0 = p->y0;
  y_1 = p->y1;
  time_stop = p->time_stop;
  g_fixed_dt = p->fixed_dt;
  x_bc = x_Periodic;
  y_bc = y_Periodic;
  g_ct_selfcheck = false;
  dx = (x_1 - x_0) / (nxPoints - 1);
  dy = (y_1 - y_0) / (nyPoints - 1);
  t = 0;
  dt = 0;
  timestep = 0;

  S.u_pri = new Grid(nx, ny); S.u_con = new Grid(nx, ny); S.u_con_n = new Grid(nx, ny);
  S.Qe = new Grid(nx, ny); S.Qe_pri = new Grid(nx, ny); S.Qs = new Grid(nx, ny);
  S.w_xL = new Grid(nx, ny); S.w_xR = new Grid(nx, ny); S.w_yL = new Grid(nx, ny);
  S.w_yR = new Grid(nx, ny); S.A = new Grid(nx, ny); S.A_n_snapshot = new Grid(nx, ny);
  S.HsA = new Tensor(RKs, nx, ny); S.HsB = new Tensor(RKs, nx, ny); S.Hs = new Tensor(RKs, nx, ny);
  S.Bx_p0 = new Array(nx, ny); S.By_0p = new Array(nx, ny); S.Bx_p0_n = new Array(nx, ny);
  S.By_0p_n = new Array(nx, ny); S.Bx = new Array(nx, ny); S.By = new Array(nx, ny);
  S.Bz = new Array(nx, ny); S.Bx_p0_Qe = new Array(nx, ny); S.By_0p_Qe = new Array(nx, ny);
  S.Bx_p0_Qs = new Array(nx, ny); S.By_0p_Qs = new Array(nx, ny);
  S.Ae = new Array(RKs, RKs); S.Ai = new Array(RKs, RKs);
  gFluxBy_p0 = new Array(nx, ny);
  gFluxBx_0p = new Array(nx, ny);
  for (Grid* g : {S.u_pri, S.u_con, S.u_con_n, S.Qe, S.Qe_pri, S.Qs, S.w_xL, S.w_xR, S.w_yL, S.w_yR, S.A,
                  S.A_n_snapshot})
    zero_grid(*g);
  for (Array* a : {S.Bx_p0, S.By_0p, S.Bx_p0_n, S.By_0p_n, S.Bx, S.By, S.Bz, S.Bx_p0_Qe, S.By_0p_Qe,
                   S.Bx_p0_Qs, S.By_0p_Qs, gFluxBy_p0, gFluxBx_0p})
    zero_array(*a);
  set_tableau();
  for (auto& row : S.snaps)
    for (auto& s : row) s.valid = false;
  S.next_stage = 0;
  S.ready = true;
  return 0;
}

// Initial data: primitive cell state (8 planes: rho, vx, vy, vz, p, Bx, By, Bz),
// face fields, vector potential (3 planes).  Mirrors main.cpp:240-244.
int ref_load_prim(const double* prim, const double* bx_face, const double* by_face, const double* A3) {
  if (!S.ready) return 1;
  grid_from_planes(*S.u_pri, prim, NUM_VARS);
  g_bc_prim = true;
  bound_cond_u(*S.u_pri);
  g_bc_prim = false;
  array_from_plane(*S.Bx_p0, bx_face);
  array_from_plane(*S.By_0p, by_face);
  bound_cond_staggered(*S.Bx_p0, 0);
  bound_cond_staggered(*S.By_0p, 1);
  upri2ucon(*S.u_con, *S.u_pri);
  grid_from_planes(*S.A, A3, 3);
  bound_cond_A(*S.A);
  t = 0;
  timestep = 0;
  S.next_stage = 0;
  return 0;
}

// One reference time step (main.cpp:335-561).  Returns the dt it used.
double ref_step(int snapshots) {
  if (!S.ready || S.next_stage != 0) return -1.0;
  S.snap_on = snapshots != 0;
  for (auto& row : S.snaps)
    for (auto& s : row) s.valid = false;
  run_step_body();
  return dt;
}

// One IMEX stage of the reference time step: the first call of a time step also
// runs the part before the stage loop (BCs, dt, GLF maxima, con<->prim), the last
// also the final con->prim.  Returns the stage index it ran, or -1 if not set up.
// RKs calls in a row give the same state as one ref_step(0).
int ref_stage(void) {
  if (!S.ready) return -1;
  const int r = S.next_stage;
  if (r == 0) run_step_pre();
  run_stage_body(r);
  if (r + 1 == RKs) {
    run_step_post();
    S.next_stage = 0;
  } else {
    S.next_stage = r + 1;
  }
  return r;
}

void ref_get_cons(double* cons8) { grid_to_planes(*S.u_con, cons8, NUM_VARS); }
void ref_get_prim(double* prim8) { grid_to_planes(*S.u_pri, prim8, NUM_VARS); }
void ref_get_faces(double* bx, double* by) {
  array_to_plane(*S.Bx_p0, bx);
  array_to_plane(*S.By_0p, by);
}
void ref_get_A(double* A3) { grid_to_planes(*S.A, A3, 3); }

// Boundary conditions (config.hpp:63-64, the x_bc / y_bc globals that main.cpp:9-233
// sets per test).  Call before ref_load_prim so that the initial ghost fills use them.
int ref_set_bc(int xbc, int ybc) {
  if (xbc < 0 || xbc > 3 || ybc < 0 || ybc > 4) return 1;
  x_bc = (x_boundary_condition)xbc;
  y_bc = (y_boundary_condition)ybc;
  return 0;
}
// The boundary normal faces that a non-periodic direction carries as degrees of freedom
// (constrained_transport.cpp:5-30): Bx_p0 at x = x_0 (index ghost_cells - 1), one value per
// row j, and By_0p at y = y_0, one per column i.  Periodic runs identify them with the
// faces at x_1 / y_1.
void ref_set_boundary_faces(const double* bx_x0, const double* by_y0) {
  for (int j = 0; j < nyCells; ++j) (*S.Bx_p0)(ghost_cells - 1, j + ghost_cells) = bx_x0[j];
  for (int i = 0; i < nxCells; ++i) (*S.By_0p)(i + ghost_cells, ghost_cells - 1) = by_y0[i];
  bound_cond_staggered(*S.Bx_p0, 0);
  bound_cond_staggered(*S.By_0p, 1);
}
void ref_get_boundary_faces(double* bx_x0, double* by_y0) {
  for (int j = 0; j < nyCells; ++j) bx_x0[j] = (*S.Bx_p0)(ghost_cells - 1, j + ghost_cells);
  for (int i = 0; i < nxCells; ++i) by_y0[i] = (*S.By_0p)(i + ghost_cells, ghost_cells - 1);
}
void ref_get_Hs(int r, double* cons8, double* hsa3, double* hsb2) {
  const int nx = nxCells, ny = nyCells;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      size_t o = i + (size_t)nx * j, N = (size_t)nx * ny;
      for (int k = 0; k < NUM_VARS; ++k) cons8[k * N + o] = (*S.Hs)(r, i + ghost_cells, j + ghost_cells, k);
      for (int k = 0; k < 3; ++k) hsa3[k * N + o] = (*S.HsA)(r, i + ghost_cells, j + ghost_cells, k);
      for (int k = 0; k < 2; ++k) hsb2[k * N + o] = (*S.HsB)(r, i + ghost_cells, j + ghost_cells, k);
    }
}

// Scalars that the step computed and the stage consumed (hidden globals).
void ref_get_scalars(double* out) {
  out[0] = dt; out[1] = adt; out[2] = B_max_x; out[3] = B_max_y; out[4] = vx_max; out[5] = vy_max;
  out[6] = a_max; out[7] = t; out[8] = ch; out[9] = v_max; out[10] = (double)timestep;
  out[11] = Mbig; out[12] = (double)g_max_floored; out[13] = g_min_p_ever;
}
void ref_set_scalars(const double* in) {
  dt = in[0]; adt = in[1]; B_max_x = in[2]; B_max_y = in[3]; vx_max = in[4]; vy_max = in[5]; a_max = in[6];
}
void ref_get_tableau(double* ae, double* ai) {
  for (int r = 0; r < RKs; ++r)
    for (int c = 0; c < RKs; ++c) {
      ae[r * RKs + c] = (*S.Ae)(r, c);
      ai[r * RKs + c] = (*S.Ai)(r, c);
    }
}

// Snapshot after sub-step `sub` of stage `rks` in the last ref_step(1).
// which: 0 u_con(8) 1 Qe(8) 2 Qs(8) 3 Bx_p0 4 By_0p 5 Bx_p0_Qs 6 By_0p_Qs 7 A(3) 8 A_s(3) 9 Fx 10 Fy
int ref_get_snapshot(int rks, int sub, int which, double* out) {
  if (rks < 0 || rks >= MAXRK || sub < 0 || sub >= NSUB) return 1;
  Snap& s = S.snaps[rks][sub];
  if (!s.valid) return 2;
  const int nx = nxCells, ny = nyCells, P = PX();
  auto grid_planes = [&](const std::vector<double>& v, int nvar) {
    for (int k = 0; k < nvar; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i)
          out[(size_t)k * nx * ny + i + (size_t)nx * j] =
              v[NUM_VARS * ((i + ghost_cells) + (size_t)(j + ghost_cells) * P) + k];
  };
  auto arr_plane = [&](const std::vector<double>& v) {
    if (v.empty()) return;
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) out[i + (size_t)nx * j] = v[(i + ghost_cells) + (size_t)(j + ghost_cells) * P];
  };
  switch (which) {
    case 0: grid_planes(s.u_con, 8); break;
    case 1: grid_planes(s.Qe, 8); break;
    case 2: grid_planes(s.Qs, 8); break;
    case 3: arr_plane(s.bx); break;
    case 4: arr_plane(s.by); break;
    case 5: arr_plane(s.bxQs); break;
    case 6: arr_plane(s.byQs); break;
    case 7: grid_planes(s.A, 3); break;
    case 8: grid_planes(s.A_s, 3); break;
    case 9: arr_plane(s.Fx); break;
    case 10: arr_plane(s.Fy); break;
    default: return 3;
  }
  return 0;
}
// The boundary-face line of a face snapshot (which = 3 Bx_p0, 5 Bx_p0_Qs: ny values at
// x = x_0; 4 By_0p, 6 By_0p_Qs: nx values at y = y_0), as ref_get_boundary_faces.
int ref_get_snapshot_boundary(int rks, int sub, int which, double* out) {
  if (rks < 0 || rks >= MAXRK || sub < 0 || sub >= NSUB) return 1;
  Snap& s = S.snaps[rks][sub];
  if (!s.valid) return 2;
  const int P = PX();
  const std::vector<double>* v = which == 3 ? &s.bx : which == 4 ? &s.by : which == 5 ? &s.bxQs
                                 : which == 6 ? &s.byQs : nullptr;
  if (!v) return 3;
  if (which == 3 || which == 5)
    for (int j = 0; j < nyCells; ++j) out[j] = (*v)[(ghost_cells - 1) + (size_t)(j + ghost_cells) * P];
  else
    for (int i = 0; i < nxCells; ++i) out[i] = (*v)[(i + ghost_cells) + (size_t)(ghost_cells - 1) * P];
  return 0;
}

// ---- single reference functions on caller-supplied state (per-kernel oracle) ----

static void load_cons(Grid& g, const double* cons8) {
  grid_from_planes(g, cons8, NUM_VARS);
  bound_cond_u(g);
}

// TVDReconstruction (reconstruction.cpp:5) of Q; outputs 4 x 8 planes (xL, xR, yL, yR).
void ref_fn_reconstruct(const double* Q8, double* out32) {
  load_cons(*S.Qe, Q8);
  TVDReconstruction(*S.Qe, *S.w_xL, *S.w_xR, *S.w_yL, *S.w_yR);
  const size_t N = (size_t)nxCells * nyCells;
  grid_to_planes(*S.w_xL, out32 + 0 * 8 * N, 8);
  grid_to_planes(*S.w_xR, out32 + 1 * 8 * N, 8);
  grid_to_planes(*S.w_yL, out32 + 2 * 8 * N, 8);
  grid_to_planes(*S.w_yR, out32 + 3 * 8 * N, 8);
}

// ShockDetector (flux.cpp:5) of Q.
void ref_fn_shock(const double* Q8, double* eta) {
  load_cons(*S.Qe, Q8);
  Array e(nxCells, nyCells);
  ShockDetector(e, *S.Qe);
  array_to_plane(e, eta);
}

// Matrix-free operators.  op: 0 Pressure L mode, 1 Pressure J mode,
// 2 Magnetic B form, 3 Magnetic A form, 4 Energy.
// For J mode, pfreeze (nx*ny) and mbig set the frozen Newton state.
void ref_fn_operator(int op, const double* ucon8, const double* Qe8, const double* Qs8, double h,
                     const double* pfreeze, double mbig, const double* x, double* Ax) {
  load_cons(*S.u_con, ucon8);
  load_cons(*S.Qe, Qe8);
  load_cons(*S.Qs, Qs8);
  const int N = nxCells * nyCells;
  const int dim = (op == 2 || op == 3) ? 3 * N : N;
  Eigen::VectorXd xv(dim), av(dim);
  for (int i = 0; i < dim; ++i) xv(i) = x[i];
  av.setZero();
  if (op == 0 || op == 1) {
    g_AX_jacobian = (op == 1);
    if (op == 1) {
      p_freeze = Eigen::VectorXd(N);
      for (int i = 0; i < N; ++i) p_freeze(i) = pfreeze[i];
      Mbig = mbig;
    }
    Pressure_Subsystem_AX(av, xv, *S.u_con, *S.Qe, *S.Qs, h);
    g_AX_jacobian = false;
  } else if (op == 2) {
    Magnetic_Subsystem_AX(av, xv, *S.u_con, *S.Qe, *S.Qs, h);
  } else if (op == 3) {
    Magnetic_Subsystem_potential_AX(av, xv, *S.u_con, *S.Qe, *S.Qs, h);
  } else {
    Energy_Subsystem_AX(av, xv, *S.u_con, *S.Qe, *S.Qs, h);
  }
  for (int i = 0; i < dim; ++i) Ax[i] = av(i);
}

// Pressure_NestedNewton (implicit_operators.cpp:625) on caller-supplied state.
void ref_fn_nested_newton(const double* ucon8, const double* Qe8, const double* Qs8, double h,
                          const double* b, double* p) {
  load_cons(*S.u_con, ucon8);
  load_cons(*S.Qe, Qe8);
  load_cons(*S.Qs, Qs8);
  const int N = nxCells * nyCells;
  Eigen::VectorXd pv(N), bv(N);
  for (int i = 0; i < N; ++i) {
    pv(i) = p[i];
    bv(i) = b[i];
  }
  Pressure_NestedNewton(pv, bv, *S.u_con, *S.Qe, *S.Qs, h, N);
  for (int i = 0; i < N; ++i) p[i] = pv(i);
}

// Full sub-steps on caller-supplied state; the state is returned in place.
// sub: 1 RusanovC_Update, 2 MagSubsystem_UpdateB/A, 3 Pressure_flux_Update,
// 4 PreSubsystem_Pressure, 5 Staggered_CT_Consistent / Unstaggered_CT_Consistent.
// For sub 3 the reconstruction of Qe is recomputed and its B slots replaced
// by cell B of u_con, exactly as main.cpp:417,447-467 do.
void ref_fn_substep(int sub, double h, int rks, double* ucon8, const double* Qe8, const double* Qs8,
                    double* bx, double* by, const double* bxQs, const double* byQs, double* A3,
                    const double* As3, double* Fx, double* Fy) {
  Grid& u_con = *S.u_con;
  load_cons(u_con, ucon8);
  load_cons(*S.Qe, Qe8);
  load_cons(*S.Qs, Qs8);
  Grid A_s(nxCells, nyCells);
  zero_grid(A_s);
  grid_from_planes(A_s, As3, 3);
  bound_cond_A(A_s);
  grid_from_planes(*S.A, A3, 3);
  bound_cond_A(*S.A);
  array_from_plane(*S.Bx_p0, bx);
  array_from_plane(*S.By_0p, by);
  bound_cond_staggered(*S.Bx_p0, 0);
  bound_cond_staggered(*S.By_0p, 1);
  array_from_plane(*S.Bx_p0_Qs, bxQs);
  array_from_plane(*S.By_0p_Qs, byQs);
  bound_cond_staggered(*S.Bx_p0_Qs, 0);
  bound_cond_staggered(*S.By_0p_Qs, 1);
  if (Fx) {
    array_from_plane(*gFluxBy_p0, Fx);
    bound_cond_array(*gFluxBy_p0);
  }
  if (Fy) {
    array_from_plane(*gFluxBx_0p, Fy);
    bound_cond_array(*gFluxBx_0p);
  }
  switch (sub) {
    case 1:
      TVDReconstruction(*S.Qe, *S.w_xL, *S.w_xR, *S.w_yL, *S.w_yR);
      RusanovC_Update(u_con, *S.Qs, *S.w_xL, *S.w_xR, *S.w_yL, *S.w_yR, h);
      break;
    case 2:
      if (magfield == PotentialA)
        MagSubsystem_UpdateA(u_con, *S.Qs, *S.Qe, *S.w_xL, *S.w_xR, *S.w_yL, *S.w_yR, *S.A, A_s, h, rks);
      else
        MagSubsystem_UpdateB(u_con, *S.Qs, *S.Qe, *S.w_xL, *S.w_xR, *S.w_yL, *S.w_yR, *S.A, h, rks);
      break;
    case 3:
      TVDReconstruction(*S.Qe, *S.w_xL, *S.w_xR, *S.w_yL, *S.w_yR);
      for (int i = 0; i < PX(); i++)
        for (int j = 0; j < PY(); j++)
          for (int k = 5; k < 8; ++k) {
            (*S.w_xL)(i, j, k) = u_con(i, j, k);
            (*S.w_xR)(i, j, k) = u_con(i, j, k);
            (*S.w_yL)(i, j, k) = u_con(i, j, k);
            (*S.w_yR)(i, j, k) = u_con(i, j, k);
          }
      if (formula == PressureFormula)
        Pressure_flux_Update(u_con, *S.Qs, *S.w_xL, *S.w_xR, *S.w_yL, *S.w_yR, h);
      else
        Energy_flux_Update(u_con, *S.Qs, *S.w_xL, *S.w_xR, *S.w_yL, *S.w_yR, h);
      break;
    case 4:
      if (formula == PressureFormula)
        PreSubsystem_Pressure(u_con, *S.Qs, *S.Qe, *S.w_xL, *S.w_xR, *S.w_yL, *S.w_yR, h, rks);
      else
        PreSubsystem_Energy(u_con, *S.Qs, *S.Qe, *S.w_xL, *S.w_xR, *S.w_yL, *S.w_yR, h, rks);
      break;
    case 5:
      if (magfield == StaggerCT)
        Staggered_CT_Consistent(u_con, *S.Bx_p0, *S.By_0p, *S.Bx_p0_Qs, *S.By_0p_Qs, h);
      else if (magfield == UnStaggerCT)
        Unstaggered_CT_Consistent(u_con, *S.A, A_s, h);
      break;
    case 6:  // legacy variants, reachable only through the commented call sites main.cpp:500,504
      if (magfield == StaggerCT)
        Staggered_CT(u_con, *S.Bx_p0, *S.By_0p, *S.Bx_p0_Qs, *S.By_0p_Qs, h);
      else if (magfield == UnStaggerCT)
        Unstaggered_CT(u_con, *S.A, A_s, h);
      break;
    default:
      break;
  }
  grid_to_planes(u_con, ucon8, 8);
  array_to_plane(*S.Bx_p0, bx);
  array_to_plane(*S.By_0p, by);
  grid_to_planes(*S.A, A3, 3);
  if (Fx) array_to_plane(*gFluxBy_p0, Fx);
  if (Fy) array_to_plane(*gFluxBx_0p, Fy);
}

// Divergence diagnostic cal_divergence_error (imex_subsystems.cpp:630).
double ref_div_error() { return cal_divergence_error(*S.u_con, *S.Bx_p0, *S.By_0p); }

// The reference's own initial data for catalogue test `test_id` (the Test ordinal of
// config.hpp:29): u_initialization (initial_conditions.cpp:5-740) and A_initial
// (constrained_transport.cpp), on the grid, domain, gamma and boundaries of ref_setup /
// ref_set_bc.  Planes as ref_get_prim / ref_get_faces / ref_get_boundary_faces / ref_get_A.
int ref_init_test(int test_id, double* prim8, double* bx, double* by, double* bx_x0, double* by_y0, double* A3) {
  if (!S.ready) return 1;
  const Test saved = test;
  test = (Test)test_id;
  u_initialization(*S.u_pri, *S.Bx_p0, *S.By_0p);
  A_initial(*S.A);
  test = saved;
  grid_to_planes(*S.u_pri, prim8, NUM_VARS);
  array_to_plane(*S.Bx_p0, bx);
  array_to_plane(*S.By_0p, by);
  ref_get_boundary_faces(bx_x0, by_y0);
  grid_to_planes(*S.A, A3, 3);
  return 0;
}

// The reference's own per-step EMF decomposition (Diagnose_CT_EMF, constrained_transport.cpp:
// 183-222, called by main.cpp:594) on the current state, its printed lines sent to `path`.
int ref_ct_diag_print(const char* path) {
  std::fflush(stdout);
  const int saved = dup(1);
  const int fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
  if (saved < 0 || fd < 0) return 1;
  dup2(fd, 1);
  Diagnose_CT_EMF(*S.u_con);
  std::fflush(stdout);
  dup2(saved, 1);
  close(saved);
  close(fd);
  return 0;
}

}  // extern "C"
