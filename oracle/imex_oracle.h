/* CPU restatement of one IMEX-RK time step of the reference 2D ideal-MHD solver.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle: tests, the smoke check and
 * the CPU-baseline leg of the benchmark call it to check the CUDA path; the
 * product never links it.  Parity of this restatement is pinned against the
 * reference's own code built by `make -C oracle ref` (oracle/_ref).
 *
 * Scope: periodic boundaries in x and y (every benchmark workload is
 * periodic), both pressure formulas' explicit fluxes, all five
 * reconstructions, the shock detector, the B-form and A-form magnetic
 * sub-systems, the pressure sub-system with the nested Newton floor (ideal
 * gas and Redlich-Kwong), GMRES(25), and the four constrained-transport
 * variants.
 *
 * Layout: interior-only SoA planes of nx*ny doubles, index i + nx*j, with
 * periodic wrap-around in place of ghost cells.  Face plane (i,j) holds Bx at
 * (i+1/2, j) / By at (i, j+1/2); the GMRES vector order equals the reference's
 * M_P / M_B maps (implicit_operators.cpp:5-139).
 *
 * The interface mirrors oracle/ref/ref_harness.cpp function for function
 * (prefix ora_ instead of ref_) so that either can serve as the checker.
 */
#ifndef IMEX_ORACLE_H
#define IMEX_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_params {
  int formula, magfield, recon, reconstate, caltimestep, add_pvisc, U_update, PressureSolver, eos_type;
  int GLF, add_bvisc, floor_on, Energy_modify, vortex_test, Pnewton_max;
  double CFL, GMREStol, gamma_plasma, p_floor, Mbig_fac, theta, Pnewton_tol, shock_kappa1;
  double m_alfa, m_b, m_R, m_cv, x0, x1, y0, y1, time_stop, fixed_dt;
} ora_params;

int ora_setup(int nx, int ny, int rks, const ora_params* p);
int ora_load_prim(const double* prim8, const double* bx, const double* by, const double* A3);
double ora_step(int snapshots);
void ora_get_cons(double* cons8);
void ora_get_prim(double* prim8);
void ora_get_faces(double* bx, double* by);
void ora_get_A(double* A3);
void ora_get_Hs(int r, double* cons8, double* hsa3, double* hsb2);
void ora_get_scalars(double* out14);
void ora_set_scalars(const double* in7);
void ora_get_tableau(double* ae, double* ai);
int ora_get_snapshot(int rks, int sub, int which, double* out);
void ora_fn_reconstruct(const double* Q8, double* out32);
void ora_fn_shock(const double* Q8, double* eta);
void ora_fn_operator(int op, const double* ucon8, const double* Qe8, const double* Qs8, double h,
                     const double* pfreeze, double mbig, const double* x, double* Ax);
void ora_fn_nested_newton(const double* ucon8, const double* Qe8, const double* Qs8, double h,
                          const double* b, double* p);
void ora_fn_substep(int sub, double h, int rks, double* ucon8, const double* Qe8, const double* Qs8,
                    double* bx, double* by, const double* bxQs, const double* byQs, double* A3,
                    const double* As3, double* Fx, double* Fy);
double ora_div_error(void);
int ora_set_bc(int x_bc, int y_bc);
void ora_set_boundary_faces(const double* bx_x0, const double* by_y0);
void ora_get_boundary_faces(double* bx_x0, double* by_y0);
int ora_get_snapshot_boundary(int rks, int sub, int which, double* out);
void ora_ct_diag(double* out16);

#ifdef __cplusplus
}
#endif
#endif
