// C ABI of libimex_b200 (include/imex_b200.h): context lifecycle, state I/O,
// the step / stage driver that replays main.cpp:335-561 on the device, the
// sub-step entry points, buffer access, statistics and diagnostics.
#include <cstdio>
#include <cstring>
#include <new>

#include "imex_internal.h"

namespace imex {

imex_status set_error(imex_ctx* ctx, imex_status s, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return s;
}
imex_status cuda_check(imex_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return IMEX_OK;
  return set_error(ctx, IMEX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---- live profile
static const char* kFamilyNames[NFAM] = {
    "step_reduce", "cons_from_prim", "stage_combine", "reconstruct", "flux_convective", "flux_pressure",
    "magnetic_rhs", "gmres_magnetic_B", "gmres_magnetic_A", "magnetic_out", "collect_mag_fluxes",
    "pressure_setup", "shock_detector", "pressure_rhs", "nested_newton", "momentum", "energy_define",
    "constrained_transport", "stage_derivative", "gmax", "gmres_pressure", "apply_operator", "mixed_refine",
    "gmres_energy", "adjoint_transposed_gmres", "adjoint_cells", "adjoint_flux", "adjoint_linear",
    "adjoint_assemble"};
const char* family_name(int fam) { return fam >= 0 && fam < NFAM ? kFamilyNames[fam] : "?"; }

static cudaEvent_t prof_event(imex_ctx* ctx) {
  if (!ctx->prof_pool.empty()) {
    cudaEvent_t e = ctx->prof_pool.back();
    ctx->prof_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
void prof_begin(imex_ctx* ctx) {
  if (!ctx->prof_on) return;
  ctx->prof_open = prof_event(ctx);
  cudaEventRecord(ctx->prof_open, ctx->stream);
}
void prof_end(imex_ctx* ctx, int fam, double bytes, int kernels) {
  ctx->kernel_launches += kernels;
  if (!ctx->prof_on || !ctx->prof_open) return;
  cudaEvent_t b = prof_event(ctx);
  cudaEventRecord(b, ctx->stream);
  ctx->prof_pending.push_back(ProfRec{ctx->prof_open, b, fam, bytes});
  ctx->prof_open = nullptr;
  if (ctx->prof_pending.size() > 4096) prof_harvest(ctx);
}
void prof_harvest(imex_ctx* ctx) {
  if (ctx->prof_pending.empty()) return;
  cudaStreamSynchronize(ctx->stream);
  for (const ProfRec& r : ctx->prof_pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      ctx->prof_ms[r.fam] += ms;
      ctx->prof_bytes[r.fam] += r.bytes;
      ctx->prof_launches[r.fam] += 1;
    }
    ctx->prof_pool.push_back(r.a);
    ctx->prof_pool.push_back(r.b);
  }
  ctx->prof_pending.clear();
}

// EOS iteration-cap flags of the two kernel translation units
imex_status eos_flag_stage(imex_ctx* ctx, int* flag, bool reset);
imex_status eos_flag_solve(imex_ctx* ctx, int* flag, bool reset);
imex_status eos_flag_stage_enqueue(imex_ctx* ctx, int* host_flag);
imex_status eos_flag_solve_enqueue(imex_ctx* ctx, int* host_flag);

namespace {

constexpr int NPSLOTS = 32;

imex_status validate(const imex_config* c, int nx, int ny, std::string& why) {
  if (nx < 4 || ny < 4) return why = "grid must be at least 4 x 4", IMEX_ERR_INVALID;
  if ((long long)nx * ny > 0x7fffffffLL) return why = "grid larger than 2^31 - 1 cells", IMEX_ERR_INVALID;
  if (c->RKs < 1 || c->RKs > kMaxRK) return why = "RKs must be 1, 2 or 3", IMEX_ERR_INVALID;
  if ((c->x_bc != IMEX_x_Periodic && c->x_bc != IMEX_x_Transmissive) ||
      (c->y_bc != IMEX_y_Periodic && c->y_bc != IMEX_y_Transmissive))
    return why = "only periodic and transmissive boundaries are implemented", IMEX_ERR_UNSUPPORTED;
  if (c->formula != IMEX_PressureFormula && c->formula != IMEX_EnergyFormula) return why = "bad formula", IMEX_ERR_INVALID;
  if (c->U_update != IMEX_DefinitionofU && c->U_update != IMEX_ConservationofU)
    return why = "U_update must be DefinitionofU or ConservationofU", IMEX_ERR_INVALID;
  if (c->recon < IMEX_NoRecon || c->recon > IMEX_WENO5) return why = "bad recon", IMEX_ERR_INVALID;
  if (c->arith != IMEX_ARITH_EXACT && c->arith != IMEX_ARITH_FAST) return why = "bad arith", IMEX_ERR_INVALID;
  if (c->magfield < IMEX_StaggerCT || c->magfield > IMEX_NoDivFree) return why = "bad magfield", IMEX_ERR_INVALID;
  if (c->gmres_restart < 1 || c->gmres_restart > 30) return why = "gmres_restart must be in 1..30", IMEX_ERR_INVALID;
  if (c->precision != IMEX_PRECISION_FP64 && c->precision != IMEX_PRECISION_MIXED)
    return why = "bad precision", IMEX_ERR_INVALID;
  if (c->precision == IMEX_PRECISION_MIXED) {
    if (!(c->mixed_inner_tol > 0.0 && c->mixed_inner_tol < 1.0))
      return why = "mixed_inner_tol must be in (0, 1)", IMEX_ERR_INVALID;
    if (c->mixed_max_refine < 1) return why = "mixed_max_refine must be at least 1", IMEX_ERR_INVALID;
    if (!(c->mixed_outer_tol >= 0.0 && c->mixed_outer_tol < 1.0))
      return why = "mixed_outer_tol must be in [0, 1)", IMEX_ERR_INVALID;
    if (c->mixed_solves & ~(IMEX_MIXED_PRESSURE | IMEX_MIXED_MAGNETIC | IMEX_MIXED_MAGNETIC_B))
      return why = "bad mixed_solves", IMEX_ERR_INVALID;
  }
  if (!(c->x_1 > c->x_0) || !(c->y_1 > c->y_0)) return why = "empty domain", IMEX_ERR_INVALID;
  return IMEX_OK;
}

template <class T>
imex_status dalloc(imex_ctx* ctx, T** p, size_t count) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, count * sizeof(T) > 0 ? count * sizeof(T) : 8);
  if (e != cudaSuccess) return cuda_check(ctx, e, "cudaMalloc");
  ctx->allocations.push_back(q);
  e = cudaMemset(q, 0, count * sizeof(T));
  if (e != cudaSuccess) return cuda_check(ctx, e, "cudaMemset");
  *p = static_cast<T*>(q);
  return IMEX_OK;
}

imex_status sync_stream(imex_ctx* ctx) { return cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync"); }

// pointer and length (in doubles) of a stage buffer
double* buffer_ptr(imex_ctx* ctx, int which, int index, size_t* count) {
  const size_t N = ctx->N;
  const int R = ctx->P.RKs;
  switch (which) {
    case IMEX_BUF_CONS: *count = 8 * N; return ctx->cons;
    case IMEX_BUF_PRIM: *count = 8 * N; return ctx->prim;
    case IMEX_BUF_CONS_N: *count = 8 * N; return ctx->cons_n;
    case IMEX_BUF_QE: *count = 8 * N; return ctx->Qe;
    case IMEX_BUF_QS: *count = 8 * N; return ctx->Qs;
    case IMEX_BUF_BX: *count = N; return ctx->bx;
    case IMEX_BUF_BY: *count = N; return ctx->by;
    case IMEX_BUF_BX_QS: *count = N; return ctx->bxQs;
    case IMEX_BUF_BY_QS: *count = N; return ctx->byQs;
    case IMEX_BUF_A: *count = 3 * N; return ctx->A;
    case IMEX_BUF_A_S: *count = 3 * N; return ctx->A_s;
    case IMEX_BUF_FLUX_X: *count = N; return ctx->Fx;
    case IMEX_BUF_FLUX_Y: *count = N; return ctx->Fy;
    case IMEX_BUF_W: *count = 32 * N; return ctx->w;
    case IMEX_BUF_HS:
      if (index < 0 || index >= R) return nullptr;
      *count = 8 * N;
      return ctx->Hs + (size_t)index * 8 * N;
    case IMEX_BUF_HSA:
      if (index < 0 || index >= R) return nullptr;
      *count = 3 * N;
      return ctx->HsA + (size_t)index * 3 * N;
    case IMEX_BUF_HSB:
      if (index < 0 || index >= R) return nullptr;
      *count = 2 * N;
      return ctx->HsB + (size_t)index * 2 * N;
    case IMEX_BUF_SHOCK: *count = N; return ctx->eta;
    case IMEX_BUF_BX_X0: *count = (size_t)ctx->ny; return ctx->bl.bx;
    case IMEX_BUF_BY_Y0: *count = (size_t)ctx->nx; return ctx->bl.by;
    case IMEX_BUF_BX_QS_X0: *count = (size_t)ctx->ny; return ctx->bl.bxQs;
    case IMEX_BUF_BY_QS_Y0: *count = (size_t)ctx->nx; return ctx->bl.byQs;
    default: return nullptr;
  }
}

imex_status read_scalars(imex_ctx* ctx) {
  cudaError_t e = cudaMemcpyAsync(ctx->h_sc, ctx->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_check(ctx, e, "scalar readback");
}
imex_status write_scalars(imex_ctx* ctx) {
  cudaError_t e = cudaMemcpyAsync(ctx->sc, ctx->h_sc, sizeof(DevScalars), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_check(ctx, e, "scalar upload");
}

// worst status recorded on the device since the last call (resets it)
// The status of the work queued so far, with one wait: the solve statistics, both EOS
// flags and (with_scalars) the step scalars come back in one round trip.
imex_status device_status(imex_ctx* ctx, bool with_scalars = false) {
  int* flags = reinterpret_cast<int*>(ctx->h_red);
  cudaError_t e = cudaMemcpyAsync(ctx->h_st, ctx->st, sizeof(DevStats), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && with_scalars)
    e = cudaMemcpyAsync(ctx->h_sc, ctx->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "status readback");
  imex_status q = eos_flag_stage_enqueue(ctx, &flags[0]);
  if (q == IMEX_OK) q = eos_flag_solve_enqueue(ctx, &flags[1]);
  if (q != IMEX_OK) return q;
  e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "status readback");
  int s = ctx->h_st->status;
  int f1 = flags[0], f2 = flags[1];
  if (f1) eos_flag_stage(ctx, &f1, true);  // clears it
  if (f2) eos_flag_solve(ctx, &f2, true);
  if ((f1 || f2) && s < IMEX_ERR_EOS) s = IMEX_ERR_EOS;
  if (s != IMEX_OK) {
    int zero = 0;
    cudaMemcpyAsync(&ctx->st->status, &zero, sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    return set_error(ctx, (imex_status)s, std::string("device reported: ") + imex_status_string((imex_status)s));
  }
  return IMEX_OK;
}

// one IMEX stage on the device (main.cpp:368-555)
imex_status stage_body(imex_ctx* ctx, int rks) {
  const DevParams& P = ctx->P;
  imex_status s;
  if ((s = launch_stage_combine(ctx, rks)) != IMEX_OK) return s;
  if ((s = launch_reconstruct(ctx, false)) != IMEX_OK) return s;
  if ((s = launch_flux_update(ctx, 0)) != IMEX_OK) return s;
  if (P.magfield == IMEX_PotentialA) s = run_mag_subsystem_A(ctx);
  else s = run_mag_subsystem_B(ctx);
  if (s != IMEX_OK) return s;
  if (P.Energy_Modify) {
    cudaError_t e = cudaMemcpyAsync(ctx->Bsave, ctx->cons + 5 * ctx->N, 3 * ctx->N * sizeof(double),
                                    cudaMemcpyDeviceToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_check(ctx, e, "Bsave");
  }
  if ((s = launch_flux_update(ctx, second_flux_form(ctx))) != IMEX_OK) return s;
  if (P.formula == IMEX_EnergyFormula) s = run_pre_subsystem_energy(ctx);
  else s = run_pre_subsystem_pressure(ctx, rks);
  if (s != IMEX_OK) return s;
  if (P.magfield == IMEX_StaggerCT) s = launch_ct(ctx, 0);
  else if (P.magfield == IMEX_UnStaggerCT) s = launch_ct(ctx, 1);
  if (s != IMEX_OK) return s;
  return launch_stage_derivative(ctx, rks);
}

}  // namespace
}  // namespace imex

using namespace imex;

namespace {
bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}
size_t op_dim(imex_ctx* ctx, int op) {
  return (op == IMEX_OP_MAGNETIC_B || op == IMEX_OP_MAGNETIC_A) ? 3 * ctx->N : ctx->N;
}
// run f(xd, bd) on device copies of host vectors when needed
template <class F>
imex_status with_device_vectors(imex_ctx* ctx, size_t n, double* x, const double* b, bool x_out, F f) {
  double* xd = x;
  const double* bd = b;
  double* tmp = nullptr;
  bool hx = x && !is_device_ptr(x), hb = b && !is_device_ptr(b);
  if (hx || hb) {
    cudaError_t e = cudaMallocAsync((void**)&tmp, 2 * n * sizeof(double), ctx->stream);
    if (e != cudaSuccess) return cuda_check(ctx, e, "temporary vectors");
    if (hx) {
      xd = tmp;
      e = cudaMemcpyAsync(xd, x, n * sizeof(double), cudaMemcpyDefault, ctx->stream);
    }
    if (hb && e == cudaSuccess) {
      bd = tmp + n;
      e = cudaMemcpyAsync(tmp + n, b, n * sizeof(double), cudaMemcpyDefault, ctx->stream);
    }
    if (e != cudaSuccess) return cuda_check(ctx, e, "vector upload");
  }
  imex_status s = f(xd, bd);
  if (s == IMEX_OK && hx && x_out) {
    cudaError_t e = cudaMemcpyAsync(x, xd, n * sizeof(double), cudaMemcpyDefault, ctx->stream);
    if (e != cudaSuccess) s = cuda_check(ctx, e, "vector download");
  }
  cudaStreamSynchronize(ctx->stream);
  if (tmp) cudaFreeAsync(tmp, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  return s;
}
imex_status ct_entry(imex_ctx* ctx, double h, int variant, int needed_magfield) {
  if (!ctx) return IMEX_ERR_INVALID;
  if (ctx->P.magfield != needed_magfield)
    return set_error(ctx, IMEX_ERR_INVALID, "CT variant does not match the configured magfield");
  imex_status s = set_h(ctx, h);
  return s != IMEX_OK ? s : launch_ct(ctx, variant);
}
}  // namespace

extern "C" {

const char* imex_status_string(imex_status s) {
  switch (s) {
    case IMEX_OK: return "ok";
    case IMEX_ERR_INVALID: return "invalid argument";
    case IMEX_ERR_UNSUPPORTED: return "unsupported configuration";
    case IMEX_ERR_CUDA: return "CUDA error";
    case IMEX_GMRES_MAXIT: return "GMRES reached its restart cap";
    case IMEX_NEWTON_MAXIT: return "nested Newton reached Pnewton_max";
    case IMEX_NONFINITE: return "non-finite value in a solve";
    case IMEX_POSITIVITY: return "pressure below theta*p_floor";
    case IMEX_ERR_SYNC: return "device barrier timed out";
    case IMEX_ERR_EOS: return "EOS Newton iteration hit its cap";
  }
  return "unknown status";
}

const char* imex_last_error(const imex_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

void imex_config_default(imex_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->caltimestep = IMEX_IMEXdt;
  c->formula = IMEX_PressureFormula;
  c->magfield = IMEX_NoDivFree;
  c->add_pvisc = IMEX_MaterialSpeedp;
  c->flux_diss = IMEX_Global_Diss;
  c->GLF = 1;
  c->add_bvisc = 1;
  c->U_update = IMEX_DefinitionofU;
  c->vortex_test = 1;
  c->RKs = 2;
  c->CFL = 0.8;
  c->recon = IMEX_Minmod;
  c->reconstate = IMEX_ConsState;
  c->x_bc = IMEX_x_Periodic;
  c->y_bc = IMEX_y_Periodic;
  c->PressureSolver = IMEX_all_correction;
  c->Energy_Modify = 0;
  c->GMREStol = 1e-14;
  c->shock_kappa1 = 0.001;
  c->floor_on = 1;
  c->p_floor = 1e-7;
  c->Mbig_fac = 1e6;
  c->theta = 0.9;
  c->Pnewton_max = 20;
  c->Pnewton_tol = 1e-8;
  c->eos_type = IMEX_IDEAL_GAS;
  c->gamma_plasma = 5.0 / 3.0;
  c->m_alfa = 0.05;
  c->m_b = 0.1;
  c->m_R = 0.4;
  c->m_cv = 1.0;
  c->x_0 = -0.5;
  c->x_1 = 0.5;
  c->y_0 = -1.0;
  c->y_1 = 1.0;
  c->time_stop = 1e30;
  c->fixed_dt = 0.0;
  c->gmres_restart = 25;
  c->gmres_max_restarts = 1000;
  c->precision = IMEX_PRECISION_FP64;
  c->mixed_inner_tol = 1e-6;
  c->mixed_max_refine = 50;
  c->mixed_solves = IMEX_MIXED_PRESSURE | IMEX_MIXED_MAGNETIC_B;
  c->mixed_outer_tol = 1e-10;
  c->arith = IMEX_ARITH_FAST;
}

imex_status imex_create(const imex_config* cfg, int nx, int ny, imex_ctx** out) {
  if (!cfg || !out) return IMEX_ERR_INVALID;
  *out = nullptr;
  std::string why;
  imex_status s = validate(cfg, nx, ny, why);
  if (s != IMEX_OK) {
    fprintf(stderr, "imex_create: %s\n", why.c_str());
    return s;
  }
  imex_ctx* ctx = new (std::nothrow) imex_ctx();
  if (!ctx) return IMEX_ERR_INVALID;
  ctx->cfg = *cfg;
  ctx->nx = nx;
  ctx->ny = ny;
  ctx->N = (size_t)nx * ny;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  ctx->device = dev;
  if (e == cudaSuccess) forget_static_scratch(dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->clock_khz, cudaDevAttrClockRate, dev);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    fprintf(stderr, "imex_create: %s\n", cudaGetErrorString(e));
    delete ctx;
    return IMEX_ERR_CUDA;
  }
  ctx->own_stream = true;
  DevParams& P = ctx->P;
  P.nx = nx;
  P.ny = ny;
  P.N = (long long)ctx->N;
  P.dx = (cfg->x_1 - cfg->x_0) / nx;
  P.dy = (cfg->y_1 - cfg->y_0) / ny;
  P.hmin = P.dy < P.dx ? P.dy : P.dx;
  P.formula = cfg->formula;
  P.magfield = cfg->magfield;
  P.recon = cfg->recon;
  P.reconstate = cfg->reconstate;
  P.vortex_minmod = cfg->vortex_test != 0;
  P.GLF = cfg->GLF;
  P.add_bvisc = cfg->add_bvisc;
  P.add_pvisc = cfg->add_pvisc;
  P.U_update = cfg->U_update;
  P.fast = cfg->arith == IMEX_ARITH_FAST;
  P.PressureSolver = cfg->PressureSolver;
  P.Energy_Modify = cfg->Energy_Modify;
  P.floor_on = cfg->floor_on;
  P.Pnewton_max = cfg->Pnewton_max;
  P.eos_type = cfg->eos_type;
  P.caltimestep = cfg->caltimestep;
  P.RKs = cfg->RKs;
  P.gamma = cfg->gamma_plasma;
  P.m_alfa = cfg->m_alfa;
  P.m_b = cfg->m_b;
  P.m_R = cfg->m_R;
  P.m_cv = cfg->m_cv;
  P.p_floor = cfg->p_floor;
  P.Mbig_fac = cfg->Mbig_fac;
  P.theta = cfg->theta;
  P.Pnewton_tol = cfg->Pnewton_tol;
  P.shock_kappa1 = cfg->shock_kappa1;
  P.GMREStol = cfg->GMREStol;
  P.CFL = cfg->CFL;
  P.time_stop = cfg->time_stop;
  P.fixed_dt = cfg->fixed_dt;
  P.xclamp = cfg->x_bc == IMEX_x_Transmissive;
  P.yclamp = cfg->y_bc == IMEX_y_Transmissive;
  P.xm = P.xclamp ? 0 : 1;
  P.xlo = P.xclamp ? 0 : nx;
  P.xhi = P.xclamp ? nx - 1 : -nx;
  P.ym = P.yclamp ? 0 : 1;
  P.ylo = P.yclamp ? 0 : ny;
  P.yhi = P.yclamp ? ny - 1 : -ny;
  {  // q = floor(n / nx) for 32-bit n: m = floor(2^32 (2^l - d) / d) + 1, l = ceil(log2 d)
     // (Granlund and Montgomery, Division by invariant integers using multiplication, 1994)
    const unsigned long long d = (unsigned long long)nx;
    int l = 0;
    while ((1ull << l) < d) ++l;
    P.nx_magic = (unsigned)((((1ull << 32) * ((1ull << l) - d)) / d) + 1ull);
    P.nx_sh1 = l < 1 ? l : 1;
    P.nx_sh2 = l > 1 ? l - 1 : 0;
  }
  P.rdx = 1.0 / P.dx;
  P.rdy = 1.0 / P.dy;

  const size_t N = ctx->N;
  const size_t R = (size_t)cfg->RKs;
  const size_t kv = (size_t)cfg->gmres_restart + 1;
  ctx->max_blocks = 4 * (ctx->num_sms > 0 ? ctx->num_sms : 148);
  s = IMEX_OK;
#define A_(ptr, n) \
  if (s == IMEX_OK) s = dalloc(ctx, &ctx->ptr, (n))
  A_(prim, 8 * N); A_(cons, 8 * N); A_(cons_n, 8 * N); A_(Qe, 8 * N); A_(Qs, 8 * N);
  A_(bx, N); A_(by, N); A_(bx_n, N); A_(by_n, N); A_(bxQe, N); A_(byQe, N); A_(bxQs, N); A_(byQs, N);
  A_(Fx, N); A_(Fy, N);
  A_(A, 3 * N); A_(A_s, 3 * N); A_(A_e, 3 * N); A_(A_snap, 3 * N);
  A_(Hs, R * 8 * N); A_(HsA, R * 3 * N); A_(HsB, R * 2 * N); A_(w, 32 * N); A_(Bsave, 3 * N);
  A_(pe, N); A_(hQe, N);
  A_(hh, N); A_(eta, N); A_(vscale, N); A_(tdiag, N); A_(vdiag, N); A_(rv, 3 * N);
  A_(irho, N);
  A_(pb, N); A_(pp, N); A_(pf, N); A_(pg, N); A_(pdp, N);
  A_(mx, 3 * N); A_(mb, 3 * N);
  if (!cfg->GLF) {
    A_(lvm, 4 * N); A_(lvp, 4 * N);
  }
  A_(chit, N); A_(Epp, N); A_(Et, N);
  const size_t lx = (size_t)ny, ly = (size_t)nx;
  A_(bline, (4 + R) * (lx + ly) + (lx + 1) + (ly + 1));
  A_(V, kv * 3 * N); A_(AV, 2 * 3 * N);
  if (cfg->precision == IMEX_PRECISION_MIXED) {
    A_(Vf, kv * 3 * N); A_(AVf, 2 * 3 * N); A_(mres, 3 * N); A_(mcor, 3 * N);
  }
  A_(partial, 2 * (size_t)ctx->max_blocks * NPSLOTS);
  ctx->partial_len = 2LL * ctx->max_blocks * NPSLOTS;
  A_(red, 64);
  A_(sc, 1); A_(st, 1); A_(sync, 1);
#undef A_
  if (s == IMEX_OK) {
    e = cudaMallocHost(&ctx->h_sc, sizeof(DevScalars));
    if (e == cudaSuccess) e = cudaMallocHost(&ctx->h_st, sizeof(DevStats));
    if (e == cudaSuccess) e = cudaMallocHost(&ctx->h_red, 64 * sizeof(double));
    if (e != cudaSuccess) s = cuda_check(ctx, e, "cudaMallocHost");
  }
  if (s == IMEX_OK) {
    BoundaryLines& L = ctx->bl;
    double* q = ctx->bline;
    L.bx = q; q += lx; L.bx_n = q; q += lx; L.bxQe = q; q += lx; L.bxQs = q; q += lx; L.hsbx = q; q += R * lx;
    L.by = q; q += ly; L.by_n = q; q += ly; L.byQe = q; q += ly; L.byQs = q; q += ly; L.hsby = q; q += R * ly;
    L.ex = q; q += lx + 1;
    L.ey = q;
    e = cudaMemsetAsync(ctx->bline, 0, ((4 + R) * (lx + ly) + (lx + 1) + (ly + 1)) * sizeof(double), ctx->stream);
    if (e != cudaSuccess) s = cuda_check(ctx, e, "boundary lines");
  }
  if (s == IMEX_OK) {
    std::memset(ctx->h_sc, 0, sizeof(DevScalars));
    s = write_scalars(ctx);
  }
  if (s == IMEX_OK) s = imex_reset_stats(ctx);
  if (s != IMEX_OK) {
    fprintf(stderr, "imex_create: %s\n", ctx->last_error.c_str());
    imex_destroy(ctx);
    return s;
  }
  *out = ctx;
  return IMEX_OK;
}

imex_status imex_destroy(imex_ctx* ctx) {
  if (!ctx) return IMEX_OK;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  prof_harvest(ctx);
  for (cudaEvent_t e : ctx->prof_pool) cudaEventDestroy(e);
  for (void* p : ctx->allocations) cudaFree(p);
  if (ctx->h_sc) cudaFreeHost(ctx->h_sc);
  if (ctx->h_st) cudaFreeHost(ctx->h_st);
  if (ctx->h_red) cudaFreeHost(ctx->h_red);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return IMEX_OK;
}

imex_status imex_set_stream(imex_ctx* ctx, void* stream) {
  if (!ctx) return IMEX_ERR_INVALID;
  cudaStreamSynchronize(ctx->stream);
  if (stream) {
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    ctx->stream = (cudaStream_t)stream;
    ctx->own_stream = false;
  } else if (!ctx->own_stream) {
    cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_check(ctx, e, "stream create");
    ctx->own_stream = true;
  }
  return IMEX_OK;
}

imex_status imex_synchronize(imex_ctx* ctx) {
  if (!ctx) return IMEX_ERR_INVALID;
  return sync_stream(ctx);
}

imex_status imex_get_config(const imex_ctx* ctx, imex_config* cfg) {
  if (!ctx || !cfg) return IMEX_ERR_INVALID;
  *cfg = ctx->cfg;
  return IMEX_OK;
}

imex_status imex_upload_prim(imex_ctx* ctx, const double* prim8, const double* bx, const double* by,
                             const double* A3) {
  if (!ctx || !prim8 || !bx || !by || !A3) return IMEX_ERR_INVALID;
  const size_t pl = ctx->N * sizeof(double);
  cudaError_t e = cudaMemcpyAsync(ctx->prim, prim8, 8 * pl, cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->bx, bx, pl, cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->by, by, pl, cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->A, A3, 3 * pl, cudaMemcpyDefault, ctx->stream);
  // boundary faces of a transmissive direction until imex_set_boundary_faces sets them: the
  // first interior face of the row / column (Bx(1/2, j), By(i, 1/2))
  if (e == cudaSuccess && ctx->P.xclamp)
    e = cudaMemcpy2DAsync(ctx->bl.bx, sizeof(double), ctx->bx, ctx->nx * sizeof(double), sizeof(double), ctx->ny,
                          cudaMemcpyDeviceToDevice, ctx->stream);
  if (e == cudaSuccess && ctx->P.yclamp)
    e = cudaMemcpyAsync(ctx->bl.by, ctx->by, ctx->nx * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "state upload");
  imex_status s = launch_cons_from_prim(ctx);
  if (s != IMEX_OK) return s;
  if ((s = read_scalars(ctx)) != IMEX_OK) return s;
  ctx->h_sc->t = 0.0;
  ctx->h_sc->timestep = 0;
  ctx->h_sc->prev_dt = 0.0;
  return write_scalars(ctx);
}

imex_status imex_upload_state(imex_ctx* ctx, const double* prim8, const double* bx, const double* by,
                              const double* A3) {
  if (!ctx || !prim8 || !bx || !by || !A3) return IMEX_ERR_INVALID;
  const size_t pl = ctx->N * sizeof(double);
  cudaError_t e = cudaMemcpyAsync(ctx->prim, prim8, 8 * pl, cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->bx, bx, pl, cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->by, by, pl, cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->A, A3, 3 * pl, cudaMemcpyDefault, ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "state upload");
  return launch_cons_from_prim(ctx);
}

imex_status imex_download_state(imex_ctx* ctx, double* cons8, double* prim8, double* bx, double* by, double* A3) {
  if (!ctx) return IMEX_ERR_INVALID;
  const size_t pl = ctx->N * sizeof(double);
  cudaError_t e = cudaSuccess;
  if (cons8 && e == cudaSuccess) e = cudaMemcpyAsync(cons8, ctx->cons, 8 * pl, cudaMemcpyDefault, ctx->stream);
  if (prim8 && e == cudaSuccess) e = cudaMemcpyAsync(prim8, ctx->prim, 8 * pl, cudaMemcpyDefault, ctx->stream);
  if (bx && e == cudaSuccess) e = cudaMemcpyAsync(bx, ctx->bx, pl, cudaMemcpyDefault, ctx->stream);
  if (by && e == cudaSuccess) e = cudaMemcpyAsync(by, ctx->by, pl, cudaMemcpyDefault, ctx->stream);
  if (A3 && e == cudaSuccess) e = cudaMemcpyAsync(A3, ctx->A, 3 * pl, cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_check(ctx, e, "state download");
}

imex_status imex_set_boundary_faces(imex_ctx* ctx, const double* bx_x0, const double* by_y0) {
  if (!ctx) return IMEX_ERR_INVALID;
  cudaError_t e = cudaSuccess;
  if (bx_x0 && ctx->P.xclamp) e = cudaMemcpyAsync(ctx->bl.bx, bx_x0, ctx->ny * sizeof(double), cudaMemcpyDefault, ctx->stream);
  if (by_y0 && ctx->P.yclamp && e == cudaSuccess)
    e = cudaMemcpyAsync(ctx->bl.by, by_y0, ctx->nx * sizeof(double), cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_check(ctx, e, "boundary faces upload");
}

imex_status imex_get_boundary_faces(imex_ctx* ctx, double* bx_x0, double* by_y0) {
  if (!ctx) return IMEX_ERR_INVALID;
  cudaError_t e = cudaSuccess;
  const size_t d = sizeof(double);
  if (bx_x0)  // a periodic x reports Bx(x_1, j), the face it identifies with x_0
    e = ctx->P.xclamp ? cudaMemcpyAsync(bx_x0, ctx->bl.bx, ctx->ny * d, cudaMemcpyDefault, ctx->stream)
                      : cudaMemcpy2DAsync(bx_x0, d, ctx->bx + (ctx->nx - 1), ctx->nx * d, d, ctx->ny, cudaMemcpyDefault,
                                          ctx->stream);
  if (by_y0 && e == cudaSuccess)
    e = cudaMemcpyAsync(by_y0, ctx->P.yclamp ? ctx->bl.by : ctx->by + (ctx->N - ctx->nx), ctx->nx * d, cudaMemcpyDefault,
                        ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_check(ctx, e, "boundary faces download");
}

imex_status imex_begin_step(imex_ctx* ctx) {
  if (!ctx) return IMEX_ERR_INVALID;
  return launch_step_prologue(ctx);
}

imex_status imex_stage(imex_ctx* ctx, int rks) {
  if (!ctx || rks < 0 || rks >= ctx->P.RKs) return IMEX_ERR_INVALID;
  return stage_body(ctx, rks);
}

imex_status imex_end_step(imex_ctx* ctx) {
  if (!ctx) return IMEX_ERR_INVALID;
  return device_status(ctx);
}

imex_status imex_step(imex_ctx* ctx, double* dt_out) {
  if (!ctx) return IMEX_ERR_INVALID;
  imex_status s = launch_step_prologue(ctx);
  for (int r = 0; s == IMEX_OK && r < ctx->P.RKs; ++r) s = stage_body(ctx, r);
  if (s != IMEX_OK) return s;
  s = device_status(ctx, dt_out != nullptr);
  if (dt_out && ctx->h_sc) *dt_out = ctx->h_sc->dt;
  return s;
}

imex_status imex_set_step_scalars(imex_ctx* ctx, const imex_step_scalars* in) {
  if (!ctx || !in) return IMEX_ERR_INVALID;
  imex_status s = read_scalars(ctx);
  if (s != IMEX_OK) return s;
  DevScalars& h = *ctx->h_sc;
  h.dt = in->dt;
  h.adt = in->adt;
  h.h = in->adt;
  h.B_max_x = in->B_max_x;
  h.B_max_y = in->B_max_y;
  h.vx_max = in->vx_max;
  h.vy_max = in->vy_max;
  h.v_max = in->v_max;
  h.a_max = in->a_max;
  h.ch = in->ch;
  h.cA_x = in->cA_x;
  h.cA_y = in->cA_y;
  h.t = in->t;
  h.timestep = in->timestep;
  return write_scalars(ctx);
}

imex_status imex_get_step_scalars(imex_ctx* ctx, imex_step_scalars* out) {
  if (!ctx || !out) return IMEX_ERR_INVALID;
  imex_status s = read_scalars(ctx);
  if (s != IMEX_OK) return s;
  const DevScalars& h = *ctx->h_sc;
  out->dt = h.dt;
  out->adt = h.adt;
  out->B_max_x = h.B_max_x;
  out->B_max_y = h.B_max_y;
  out->vx_max = h.vx_max;
  out->vy_max = h.vy_max;
  out->v_max = h.v_max;
  out->a_max = h.a_max;
  out->ch = h.ch;
  out->cA_x = h.cA_x;
  out->cA_y = h.cA_y;
  out->t = h.t;
  out->timestep = h.timestep;
  return IMEX_OK;
}

// ---- sub-steps
imex_status imex_stage_combine(imex_ctx* ctx, int rks) {
  if (!ctx || rks < 0 || rks >= ctx->P.RKs) return IMEX_ERR_INVALID;
  return launch_stage_combine(ctx, rks);
}
imex_status imex_TVDReconstruction(imex_ctx* ctx) {
  if (!ctx) return IMEX_ERR_INVALID;
  return launch_reconstruct(ctx, true);
}
imex_status imex_RusanovC_Update(imex_ctx* ctx, double h, int rks) {
  if (!ctx) return IMEX_ERR_INVALID;
  (void)rks;
  imex_status s = set_h(ctx, h);
  return s != IMEX_OK ? s : launch_flux_update(ctx, 0);
}
imex_status imex_MagSubsystem_UpdateB(imex_ctx* ctx, double h, int rks) {
  if (!ctx) return IMEX_ERR_INVALID;
  (void)rks;
  imex_status s = set_h(ctx, h);
  if (s == IMEX_OK) s = launch_qe_derived(ctx);
  if (s == IMEX_OK) s = run_mag_subsystem_B(ctx);
  return s != IMEX_OK ? s : device_status(ctx);
}
imex_status imex_MagSubsystem_UpdateA(imex_ctx* ctx, double h, int rks) {
  if (!ctx) return IMEX_ERR_INVALID;
  (void)rks;
  imex_status s = set_h(ctx, h);
  if (s == IMEX_OK) s = launch_qe_derived(ctx);
  ctx->gmax_ready = false;  // Qs is the caller's: take its maxima
  if (s == IMEX_OK) s = run_mag_subsystem_A(ctx);
  return s != IMEX_OK ? s : device_status(ctx);
}
imex_status imex_Pressure_flux_Update(imex_ctx* ctx, double h, int rks) {
  if (!ctx) return IMEX_ERR_INVALID;
  (void)rks;
  imex_status s = set_h(ctx, h);
  return s != IMEX_OK ? s : launch_flux_update(ctx, 1);
}
imex_status imex_PreSubsystem_Pressure(imex_ctx* ctx, double h, int rks) {
  if (!ctx) return IMEX_ERR_INVALID;
  imex_status s = set_h(ctx, h);
  if (s == IMEX_OK) s = launch_qe_derived(ctx);
  if (s == IMEX_OK) s = run_pre_subsystem_pressure(ctx, rks);
  return s != IMEX_OK ? s : device_status(ctx);
}
imex_status imex_Energy_flux_Update(imex_ctx* ctx, double h, int rks) {
  if (!ctx) return IMEX_ERR_INVALID;
  (void)rks;
  imex_status s = set_h(ctx, h);
  return s != IMEX_OK ? s : launch_flux_update(ctx, 2);
}
imex_status imex_PreSubsystem_Energy(imex_ctx* ctx, double h, int rks) {
  if (!ctx) return IMEX_ERR_INVALID;
  (void)rks;
  imex_status s = set_h(ctx, h);
  if (s == IMEX_OK) s = run_pre_subsystem_energy(ctx);
  return s != IMEX_OK ? s : device_status(ctx);
}
imex_status imex_Staggered_CT_Consistent(imex_ctx* ctx, double h, int) { return ct_entry(ctx, h, 0, IMEX_StaggerCT); }
imex_status imex_Unstaggered_CT_Consistent(imex_ctx* ctx, double h, int) {
  return ct_entry(ctx, h, 1, IMEX_UnStaggerCT);
}
imex_status imex_Staggered_CT(imex_ctx* ctx, double h, int) { return ct_entry(ctx, h, 2, IMEX_StaggerCT); }
imex_status imex_Unstaggered_CT(imex_ctx* ctx, double h, int) { return ct_entry(ctx, h, 3, IMEX_UnStaggerCT); }
imex_status imex_stage_derivative(imex_ctx* ctx, int rks) {
  if (!ctx || rks < 0 || rks >= ctx->P.RKs) return IMEX_ERR_INVALID;
  return launch_stage_derivative(ctx, rks);
}

// ---- buffers
imex_status imex_buffer_count(const imex_ctx* ctx, int which, size_t* n) {
  if (!ctx || !n) return IMEX_ERR_INVALID;
  double* p = buffer_ptr(const_cast<imex_ctx*>(ctx), which, 0, n);
  return p ? IMEX_OK : IMEX_ERR_INVALID;
}
imex_status imex_set_buffer(imex_ctx* ctx, int which, int index, const double* src) {
  if (!ctx || !src) return IMEX_ERR_INVALID;
  size_t n = 0;
  double* p = buffer_ptr(ctx, which, index, &n);
  if (!p) return set_error(ctx, IMEX_ERR_INVALID, "bad buffer id or index");
  cudaError_t e = cudaMemcpyAsync(p, src, n * sizeof(double), cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_check(ctx, e, "set buffer");
}
imex_status imex_get_buffer(imex_ctx* ctx, int which, int index, double* dst) {
  if (!ctx || !dst) return IMEX_ERR_INVALID;
  size_t n = 0;
  double* p = buffer_ptr(ctx, which, index, &n);
  if (!p) return set_error(ctx, IMEX_ERR_INVALID, "bad buffer id or index");
  cudaError_t e = cudaMemcpyAsync(dst, p, n * sizeof(double), cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_check(ctx, e, "get buffer");
}

// ---- operators and solves
imex_status imex_prepare_operator(imex_ctx* ctx, int op, double h) {
  if (!ctx || op < 0 || op > IMEX_OP_ENERGY) return IMEX_ERR_INVALID;
  return prepare_operator(ctx, op, h);
}
imex_status imex_set_newton_state(imex_ctx* ctx, const double* p_freeze, double mbig) {
  if (!ctx || !p_freeze) return IMEX_ERR_INVALID;
  return set_newton_state(ctx, p_freeze, mbig);
}
imex_status imex_apply_operator(imex_ctx* ctx, int op, const double* x, double* Ax) {
  if (!ctx || !x || !Ax) return IMEX_ERR_INVALID;
  const size_t n = op_dim(ctx, op);
  return with_device_vectors(ctx, n, Ax, x, true,
                             [&](double* axd, const double* xd) { return apply_operator(ctx, op, xd, axd); });
}
imex_status imex_gmres(imex_ctx* ctx, int op, double* x, const double* b, imex_solve_stats* stats) {
  if (!ctx || !x || !b) return IMEX_ERR_INVALID;
  const size_t n = op_dim(ctx, op);
  imex_status s = with_device_vectors(ctx, n, x, b, true,
                                      [&](double* xd, const double* bd) { return run_gmres(ctx, op, xd, bd); });
  if (s != IMEX_OK) return s;
  s = device_status(ctx);
  if (stats) imex_get_stats(ctx, stats);
  return s;
}
imex_status imex_gmres_noalloc(imex_ctx* ctx, int op, double* x, const double* b, imex_solve_stats* stats) {
  if (!ctx || !x || !b) return IMEX_ERR_INVALID;
  unsigned char* base = nullptr;
  imex_status s = static_scratch(ctx, &base);
  if (s != IMEX_OK) return s;
  s = run_gmres_noalloc(ctx, op, x, b, base, kStaticScratchBytes);
  if (s != IMEX_OK) return s;
  s = device_status(ctx);
  if (stats) imex_get_stats(ctx, stats);
  return s;
}
imex_status imex_pressure_nested_newton(imex_ctx* ctx, double* p, const double* b, imex_solve_stats* stats) {
  if (!ctx || !p || !b) return IMEX_ERR_INVALID;
  imex_status s = with_device_vectors(ctx, ctx->N, p, b, true,
                                      [&](double* pd, const double* bd) { return run_nested_newton(ctx, pd, bd); });
  if (s != IMEX_OK) return s;
  s = device_status(ctx);
  if (stats) imex_get_stats(ctx, stats);
  return s;
}
imex_status imex_shock_detector(imex_ctx* ctx, const double* Q8, double* eta) {
  if (!ctx || !Q8 || !eta) return IMEX_ERR_INVALID;
  // the reconstruction buffer (32 planes) doubles as scratch: Q in planes 0-7, eta in plane 8
  double* q = ctx->w;
  double* e8 = ctx->w + 8 * ctx->N;
  cudaError_t e = cudaMemcpyAsync(q, Q8, 8 * ctx->N * sizeof(double), cudaMemcpyDefault, ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "shock input");
  imex_status s = launch_shock(ctx, q, e8);
  if (s != IMEX_OK) return s;
  e = cudaMemcpyAsync(eta, e8, ctx->N * sizeof(double), cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_check(ctx, e, "shock output");
}

// ---- statistics and diagnostics
imex_status imex_get_stats(imex_ctx* ctx, imex_solve_stats* out) {
  if (!ctx || !out) return IMEX_ERR_INVALID;
  cudaError_t e = cudaMemcpyAsync(ctx->h_st, ctx->st, sizeof(DevStats), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "stats readback");
  const DevStats& d = *ctx->h_st;
  out->gmres_solves = d.gmres_solves;
  out->gmres_iters = d.gmres_iters;
  out->gmres_restarts = d.gmres_restarts;
  out->newton_iters = d.newton_iters;
  out->max_floored = d.max_floored;
  out->refine_sweeps = d.refine_sweeps;
  out->last_residual = d.last_residual;
  out->min_p = d.min_p;
  out->status = d.status;
  return IMEX_OK;
}
imex_status imex_reset_stats(imex_ctx* ctx) {
  if (!ctx) return IMEX_ERR_INVALID;
  std::memset(ctx->h_st, 0, sizeof(DevStats));
  ctx->h_st->min_p = 1e300;
  cudaError_t e = cudaMemcpyAsync(ctx->st, ctx->h_st, sizeof(DevStats), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_check(ctx, e, "stats reset");
}
imex_status imex_divergence(imex_ctx* ctx, double* face_l2, double* wrapped_l2, double* ref_l2, double* cell_inf) {
  if (!ctx) return IMEX_ERR_INVALID;
  double o[4];
  imex_status s = launch_divergence(ctx, o);
  if (s != IMEX_OK) return s;
  if (face_l2) *face_l2 = o[0];
  if (wrapped_l2) *wrapped_l2 = o[1];
  if (ref_l2) *ref_l2 = o[2];
  if (cell_inf) *cell_inf = o[3];
  return IMEX_OK;
}
imex_status imex_profile_enable(imex_ctx* ctx, int on) {
  if (!ctx) return IMEX_ERR_INVALID;
  prof_harvest(ctx);
  for (int f = 0; f < NFAM; ++f) {
    ctx->prof_ms[f] = 0.0;
    ctx->prof_bytes[f] = 0.0;
    ctx->prof_launches[f] = 0;
  }
  static const double zeros[NFAM] = {};
  cudaError_t e = cudaMemcpyAsync(ctx->st->alg_bytes, zeros, sizeof(zeros), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  ctx->prof_on = on != 0;
  return cuda_check(ctx, e, "profile reset");
}
imex_status imex_kernel_launch_count(const imex_ctx* ctx, long long* count) {
  if (!ctx || !count) return IMEX_ERR_INVALID;
  *count = ctx->kernel_launches;
  return IMEX_OK;
}
imex_status imex_profile_read(imex_ctx* ctx, imex_kernel_profile* out, int max, int* count) {
  if (!ctx || !out || !count) return IMEX_ERR_INVALID;
  prof_harvest(ctx);
  double dev[NFAM];
  cudaError_t e = cudaMemcpyAsync(dev, ctx->st->alg_bytes, sizeof(dev), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "profile readback");
  int n = 0;
  for (int f = 0; f < NFAM && n < max; ++f) {
    if (ctx->prof_launches[f] == 0) continue;
    imex_kernel_profile& r = out[n++];
    std::memset(&r, 0, sizeof(r));
    std::strncpy(r.name, family_name(f), sizeof(r.name) - 1);
    r.launches = ctx->prof_launches[f];
    r.total_ms = ctx->prof_ms[f];
    r.alg_bytes = ctx->prof_bytes[f] + dev[f];
  }
  *count = n;
  return IMEX_OK;
}
imex_status imex_selftest_barrier(imex_ctx* ctx, int iterations, int phantom_blocks, double timeout_s,
                                  double* us_per_barrier) {
  if (!ctx || iterations < 0 || phantom_blocks < 0 || !(timeout_s > 0.0) || timeout_s > 60.0) return IMEX_ERR_INVALID;
  imex_status s = run_barrier_selftest(ctx, iterations, phantom_blocks, timeout_s, us_per_barrier);
  return s != IMEX_OK ? s : device_status(ctx);
}
imex_status imex_selftest_fp64(imex_ctx* ctx, double* dfma_per_s, double* ddiv_per_s) {
  if (!ctx) return IMEX_ERR_INVALID;
  return run_fp64_selftest(ctx, dfma_per_s, ddiv_per_s);
}
imex_status imex_set_barrier_timeout(imex_ctx* ctx, double seconds) {
  if (!ctx || !(seconds > 0.0) || seconds > 600.0) return IMEX_ERR_INVALID;
  ctx->barrier_timeout_s = seconds;
  return IMEX_OK;
}
imex_status imex_min_pressure(imex_ctx* ctx, double* pmin) {
  if (!ctx || !pmin) return IMEX_ERR_INVALID;
  return launch_min_pressure(ctx, pmin);
}

}  // extern "C"
