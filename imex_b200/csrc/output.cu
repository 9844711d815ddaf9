// Output formats and run diagnostics (the reference's main.cpp:560-721 and output.cpp):
//   * imex_diagnostics: the per-step quantities the reference prints and records
//     (cal_divergence_error, the max central div B, imex_dt / fully_dt, and the DIAG line's
//     min internal energy and where, mass, internal energy, max magnetic energy);
//   * a legacy-VTK rectilinear-grid writer with the reference's 13 cell fields, written
//     with the node coordinates the header declares (nx + 1, ny + 1) and the interior cells
//     only, at full precision (output.cpp:127-192 declares nx + 1 coordinates but prints nx
//     cell centres, and indexes cells from the ghost corner);
//   * the final-state field files RK_<field>.dat (x y value per cell, main.cpp:598-695) and
//     the step histories RK_div_error.dat, RK_B_inf.dat, RK_dt_comp.dat (main.cpp:697-710),
//     at full precision instead of the stream default of six digits;
//   * a binary state file (primitive planes, faces, A and the step scalars) from which a run
//     continues bit for bit.
// The writers have host-only entry points (imex_*_host) that need no GPU.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "device_common.cuh"
#include "imex_internal.h"

namespace imex {
namespace {

constexpr int kDT = 256;

// block partials of (sum rho, sum e, min e, max |B|^2 / 2) over the cells (main.cpp:565-573)
__global__ void k_diag(DevParams P, const double* __restrict__ u, double* __restrict__ partial) {
  __shared__ double sh[4][kDT / 32];
  const long long N = P.N;
  double mass = 0.0, intE = 0.0, emin = INFINITY, mmax = -INFINITY;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N; n += (long long)gridDim.x * blockDim.x) {
    const double rho = u[n];
    const double k = 0.5 * (u[N + n] * u[N + n] + u[2 * N + n] * u[2 * N + n] + u[3 * N + n] * u[3 * N + n]) / rho;
    const double m = 0.5 * (u[5 * N + n] * u[5 * N + n] + u[6 * N + n] * u[6 * N + n] + u[7 * N + n] * u[7 * N + n]);
    const double e = u[4 * N + n] - k - m;
    mass += rho;
    intE += e;
    emin = fmin(emin, e);
    mmax = fmax(mmax, m);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mass += __shfl_xor_sync(0xffffffffu, mass, o);
    intE += __shfl_xor_sync(0xffffffffu, intE, o);
    emin = fmin(emin, __shfl_xor_sync(0xffffffffu, emin, o));
    mmax = fmax(mmax, __shfl_xor_sync(0xffffffffu, mmax, o));
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    sh[0][w] = mass;
    sh[1][w] = intE;
    sh[2][w] = emin;
    sh[3][w] = mmax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < kDT / 32; ++q) {
      mass += sh[0][q];
      intE += sh[1][q];
      emin = fmin(emin, sh[2][q]);
      mmax = fmax(mmax, sh[3][q]);
    }
    partial[4 * blockIdx.x + 0] = mass;
    partial[4 * blockIdx.x + 1] = intE;
    partial[4 * blockIdx.x + 2] = emin;
    partial[4 * blockIdx.x + 3] = mmax;
  }
}
// first cell (i outer, j inner as the reference's loop) where e attains its minimum
__global__ void k_diag_argmin(DevParams P, const double* __restrict__ u, double emin, unsigned long long* idx) {
  const long long N = P.N;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  const double rho = u[n];
  const double k = 0.5 * (u[N + n] * u[N + n] + u[2 * N + n] * u[2 * N + n] + u[3 * N + n] * u[3 * N + n]) / rho;
  const double m = 0.5 * (u[5 * N + n] * u[5 * N + n] + u[6 * N + n] * u[6 * N + n] + u[7 * N + n] * u[7 * N + n]);
  if (u[4 * N + n] - k - m == emin) {
    const long long i = n % P.nx, j = n / P.nx;
    atomicMin(idx, (unsigned long long)(i * P.ny + j));
  }
}
// Redlich-Kwong temperature of the primitive state (RK_T.dat, main.cpp:712-721)
__global__ void k_temperature(DevParams P, const double* __restrict__ prim, double* __restrict__ T) {
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n < P.N) T[n] = rk_T_from_rho_p(P, prim[n], prim[4 * P.N + n]);
}

constexpr char kMagic[8] = {'I', 'M', 'E', 'X', 'S', 'T', 'A', 'T'};
struct StateHeader {
  char magic[8];
  int version, nx, ny, timestep;
  double t, prev_dt, dt, x0, x1, y0, y1;
};

imex_status host_download(imex_ctx* ctx, std::vector<double>& cons, std::vector<double>& prim) {
  cons.resize(8 * ctx->N);
  prim.resize(8 * ctx->N);
  return imex_download_state(ctx, cons.data(), prim.data(), nullptr, nullptr, nullptr);
}
imex_status io_error(imex_ctx* ctx, const std::string& what, const char* path) {
  return set_error(ctx, IMEX_ERR_INVALID, what + " '" + path + "': " + strerror(errno));
}

}  // namespace
}  // namespace imex

using namespace imex;

extern "C" {

// ---- host-only writers
int imex_vtk_write_host(const char* path, int nx, int ny, double x0, double y0, double dx, double dy, double t,
                        int cycle, const double* cons8, const double* prim8) {
  if (!path || !cons8 || !prim8 || nx < 1 || ny < 1) return IMEX_ERR_INVALID;
  FILE* f = fopen(path, "w");
  if (!f) return IMEX_ERR_INVALID;
  const size_t N = (size_t)nx * ny;
  fprintf(f, "# vtk DataFile Version 3.0\nvtk output\nASCII\nDATASET RECTILINEAR_GRID\n");
  fprintf(f, "FIELD FieldData 2\nCYCLE 1 1 int\n%d\nTIME 1 1 double\n%.17g\n", cycle, t);
  fprintf(f, "DIMENSIONS %d %d 1\n", nx + 1, ny + 1);
  fprintf(f, "X_COORDINATES %d double\n", nx + 1);
  for (int i = 0; i <= nx; ++i) fprintf(f, "%.17g%c", x0 + i * dx, i == nx ? '\n' : ' ');
  fprintf(f, "Y_COORDINATES %d double\n", ny + 1);
  for (int j = 0; j <= ny; ++j) fprintf(f, "%.17g%c", y0 + j * dy, j == ny ? '\n' : ' ');
  fprintf(f, "Z_COORDINATES 1 double\n0\n");
  fprintf(f, "CELL_DATA %zu\n", N);
  // the reference's variable list (output.cpp:300-312): conserved 0-7, velX/Y/Z and p, |B|
  static const char* names[13] = {"rho", "mom_X", "mom_Y", "mom_Z", "U", "B_X", "B_Y", "B_Z",
                                  "velX", "velY", "velZ", "p", "B"};
  fprintf(f, "FIELD FieldData 13\n");
  for (int v = 0; v < 13; ++v) {
    fprintf(f, "%s 1 %zu double\n", names[v], N);
    for (int j = 0; j < ny; ++j) {
      for (int i = 0; i < nx; ++i) {
        const size_t c = (size_t)i + (size_t)nx * j;
        double val;
        if (v < 8) val = cons8[v * N + c];
        else if (v < 12) val = prim8[(v - 7) * N + c];
        else val = sqrt(cons8[5 * N + c] * cons8[5 * N + c] + cons8[6 * N + c] * cons8[6 * N + c] +
                        cons8[7 * N + c] * cons8[7 * N + c]);
        fprintf(f, "%.17g%c", val, i == nx - 1 ? '\n' : ' ');
      }
    }
  }
  return fclose(f) == 0 ? IMEX_OK : IMEX_ERR_INVALID;
}

// "x y value" per cell, x outer and y inner as the reference (main.cpp:598-606)
int imex_dat_write_host(const char* path, int nx, int ny, double x0, double y0, double dx, double dy,
                        const double* plane) {
  if (!path || !plane || nx < 1 || ny < 1) return IMEX_ERR_INVALID;
  FILE* f = fopen(path, "w");
  if (!f) return IMEX_ERR_INVALID;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      fprintf(f, "%.17g %.17g %.17g\n", x0 + dx * (i + 0.5), y0 + dy * (j + 0.5), plane[(size_t)i + (size_t)nx * j]);
  return fclose(f) == 0 ? IMEX_OK : IMEX_ERR_INVALID;
}

// "timestep value" per line (main.cpp:697-710)
int imex_history_write_host(const char* path, int n, const int* steps, const double* values) {
  if (!path || n < 0 || (n > 0 && (!steps || !values))) return IMEX_ERR_INVALID;
  FILE* f = fopen(path, "w");
  if (!f) return IMEX_ERR_INVALID;
  for (int k = 0; k < n; ++k) fprintf(f, "%d %.17g\n", steps[k], values[k]);
  return fclose(f) == 0 ? IMEX_OK : IMEX_ERR_INVALID;
}

// ---- on a context
imex_status imex_ct_emf_diagnostics(imex_ctx* ctx, double* out16) {
  if (!ctx || !out16) return IMEX_ERR_INVALID;
  return launch_ct_diag(ctx, out16);
}

imex_status imex_diagnostics(imex_ctx* ctx, imex_diagnostics_t* d) {
  if (!ctx || !d) return IMEX_ERR_INVALID;
  const DevParams& P = ctx->P;
  double face_l2 = 0, wrapped_l2 = 0, ref_l2 = 0, inf = 0;
  imex_status s = imex_divergence(ctx, &face_l2, &wrapped_l2, &ref_l2, &inf);
  if (s != IMEX_OK) return s;
  int nblk = (int)((P.N + kDT - 1) / kDT);
  if (nblk > ctx->max_blocks) nblk = ctx->max_blocks;
  k_diag<<<nblk, kDT, 0, ctx->stream>>>(P, ctx->cons, ctx->partial);
  std::vector<double> part(4 * (size_t)nblk);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(part.data(), ctx->partial, part.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "diagnostics");
  double mass = 0, intE = 0, emin = INFINITY, mmax = -INFINITY;
  for (int b = 0; b < nblk; ++b) {
    mass += part[4 * b];
    intE += part[4 * b + 1];
    emin = fmin(emin, part[4 * b + 2]);
    mmax = fmax(mmax, part[4 * b + 3]);
  }
  unsigned long long* idx = reinterpret_cast<unsigned long long*>(ctx->red);
  const unsigned long long none = ~0ull;
  e = cudaMemcpyAsync(idx, &none, sizeof(none), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) {
    k_diag_argmin<<<(unsigned)((P.N + kDT - 1) / kDT), kDT, 0, ctx->stream>>>(P, ctx->cons, emin, idx);
    e = cudaGetLastError();
  }
  unsigned long long at = none;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&at, idx, sizeof(at), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "diagnostics");
  ctx->kernel_launches += 2;
  e = cudaMemcpyAsync(ctx->h_sc, ctx->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "diagnostics");
  const DevScalars& sc = *ctx->h_sc;
  memset(d, 0, sizeof(*d));
  d->timestep = sc.timestep;
  d->t = sc.t;
  d->dt = sc.dt;
  d->div_error = P.magfield == IMEX_StaggerCT ? face_l2 : ref_l2;
  d->B_inf = inf;
  // imex_dt / fully_dt of caldt (timestep.cpp:56-57): the dt's speed over the fast speed
  const double full = P.CFL * 1 / (2 * sc.ch / fmin(P.dx, P.dy));
  double a_dt;
  if (P.caltimestep == IMEX_Fullydt) a_dt = sc.ch;
  else if (P.caltimestep == IMEX_Alfvendt) a_dt = sc.timestep < 2 ? sc.ch : sc.cA;
  else a_dt = sc.timestep < 2 ? sc.ch : sc.v_max;
  d->dt_comp = (P.CFL * 1 / (2 * a_dt / fmin(P.dx, P.dy))) / full;
  d->emin = emin;
  if (at != none) {
    const long long i = (long long)(at / (unsigned long long)P.ny), j = (long long)(at % (unsigned long long)P.ny);
    d->emin_x = ctx->cfg.x_0 + (i + 0.5) * P.dx;
    d->emin_y = ctx->cfg.y_0 + (j + 0.5) * P.dy;
  }
  d->mass = mass * P.dx * P.dy;
  d->intE = intE * P.dx * P.dy;
  d->magE_max = mmax;
  return IMEX_OK;
}

imex_status imex_write_vtk(imex_ctx* ctx, const char* path, int cycle) {
  if (!ctx || !path) return IMEX_ERR_INVALID;
  std::vector<double> cons, prim;
  imex_status s = host_download(ctx, cons, prim);
  if (s != IMEX_OK) return s;
  imex_step_scalars sc{};
  if ((s = imex_get_step_scalars(ctx, &sc)) != IMEX_OK) return s;
  const DevParams& P = ctx->P;
  if (imex_vtk_write_host(path, ctx->nx, ctx->ny, ctx->cfg.x_0, ctx->cfg.y_0, P.dx, P.dy, sc.t, cycle, cons.data(),
                          prim.data()) != IMEX_OK)
    return io_error(ctx, "cannot write", path);
  return IMEX_OK;
}

imex_status imex_write_fields_dat(imex_ctx* ctx, const char* dir) {
  if (!ctx || !dir) return IMEX_ERR_INVALID;
  std::vector<double> cons, prim;
  imex_status s = host_download(ctx, cons, prim);
  if (s != IMEX_OK) return s;
  const DevParams& P = ctx->P;
  const size_t N = ctx->N;
  std::vector<double> vmag(N);
  for (size_t c = 0; c < N; ++c) vmag[c] = sqrt(prim[N + c] * prim[N + c] + prim[2 * N + c] * prim[2 * N + c]);
  struct Out {
    const char* name;
    const double* plane;
  } outs[] = {{"RK_rho.dat", cons.data()},         {"RK_vx.dat", prim.data() + N},
              {"RK_vy.dat", prim.data() + 2 * N},   {"RK_E.dat", cons.data() + 4 * N},
              {"RK_p.dat", prim.data() + 4 * N},    {"RK_Bx.dat", prim.data() + 5 * N},
              {"RK_By.dat", prim.data() + 6 * N},   {"RK_Bz.dat", prim.data() + 7 * N},
              {"RK_v_mag.dat", vmag.data()}};
  for (const Out& o : outs) {
    const std::string path = std::string(dir) + "/" + o.name;
    if (imex_dat_write_host(path.c_str(), ctx->nx, ctx->ny, ctx->cfg.x_0, ctx->cfg.y_0, P.dx, P.dy, o.plane) !=
        IMEX_OK)
      return io_error(ctx, "cannot write", path.c_str());
  }
  if (P.eos_type == IMEX_REDLICH_KWONG) {
    double* T = nullptr;
    cudaError_t e = cudaMalloc(&T, N * sizeof(double));
    std::vector<double> hT(N);
    if (e == cudaSuccess) {
      k_temperature<<<(unsigned)((N + kDT - 1) / kDT), kDT, 0, ctx->stream>>>(P, ctx->prim, T);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(hT.data(), T, N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (T) cudaFree(T);
    if (e != cudaSuccess) return cuda_check(ctx, e, "temperature");
    const std::string path = std::string(dir) + "/RK_T.dat";
    if (imex_dat_write_host(path.c_str(), ctx->nx, ctx->ny, ctx->cfg.x_0, ctx->cfg.y_0, P.dx, P.dy, hT.data()) !=
        IMEX_OK)
      return io_error(ctx, "cannot write", path.c_str());
  }
  return IMEX_OK;
}

imex_status imex_save_state_file(imex_ctx* ctx, const char* path) {
  if (!ctx || !path) return IMEX_ERR_INVALID;
  const size_t N = ctx->N;
  std::vector<double> buf((8 + 1 + 1 + 3) * N);
  imex_status s = imex_download_state(ctx, nullptr, buf.data(), buf.data() + 8 * N, buf.data() + 9 * N,
                                      buf.data() + 10 * N);
  if (s != IMEX_OK) return s;
  cudaError_t e = cudaMemcpyAsync(ctx->h_sc, ctx->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "state scalars");
  // a transmissive run appends its boundary normal faces (ny values of Bx on x_0, nx of By
  // on y_0) and marks the file version 2
  const bool lines = ctx->P.xclamp || ctx->P.yclamp;
  if (lines) {
    buf.resize(buf.size() + ctx->ny + ctx->nx);
    s = imex_get_boundary_faces(ctx, buf.data() + 13 * N, buf.data() + 13 * N + ctx->ny);
    if (s != IMEX_OK) return s;
  }
  StateHeader h{};
  memcpy(h.magic, kMagic, 8);
  h.version = lines ? 2 : 1;
  h.nx = ctx->nx;
  h.ny = ctx->ny;
  h.timestep = ctx->h_sc->timestep;
  h.t = ctx->h_sc->t;
  h.prev_dt = ctx->h_sc->prev_dt;
  h.dt = ctx->h_sc->dt;
  h.x0 = ctx->cfg.x_0;
  h.x1 = ctx->cfg.x_1;
  h.y0 = ctx->cfg.y_0;
  h.y1 = ctx->cfg.y_1;
  FILE* f = fopen(path, "wb");
  if (!f) return io_error(ctx, "cannot write", path);
  bool ok = fwrite(&h, sizeof(h), 1, f) == 1 && fwrite(buf.data(), sizeof(double), buf.size(), f) == buf.size();
  ok = (fclose(f) == 0) && ok;
  return ok ? IMEX_OK : io_error(ctx, "cannot write", path);
}

imex_status imex_load_state_file(imex_ctx* ctx, const char* path) {
  if (!ctx || !path) return IMEX_ERR_INVALID;
  FILE* f = fopen(path, "rb");
  if (!f) return io_error(ctx, "cannot read", path);
  StateHeader h{};
  const size_t N = ctx->N;
  std::vector<double> buf((8 + 1 + 1 + 3) * N);
  bool ok = fread(&h, sizeof(h), 1, f) == 1;
  if (ok && (memcmp(h.magic, kMagic, 8) != 0 || (h.version != 1 && h.version != 2) || h.nx != ctx->nx ||
             h.ny != ctx->ny)) {
    fclose(f);
    return set_error(ctx, IMEX_ERR_INVALID, std::string("'") + path + "' is not a state file of this grid");
  }
  if (h.version == 2) buf.resize(buf.size() + ctx->ny + ctx->nx);
  ok = ok && fread(buf.data(), sizeof(double), buf.size(), f) == buf.size();
  fclose(f);
  if (!ok) return set_error(ctx, IMEX_ERR_INVALID, std::string("short state file '") + path + "'");
  imex_status s = imex_upload_prim(ctx, buf.data(), buf.data() + 8 * N, buf.data() + 9 * N, buf.data() + 10 * N);
  if (s == IMEX_OK && h.version == 2)
    s = imex_set_boundary_faces(ctx, buf.data() + 13 * N, buf.data() + 13 * N + ctx->ny);
  if (s != IMEX_OK) return s;
  cudaError_t e = cudaMemcpyAsync(ctx->h_sc, ctx->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_check(ctx, e, "state scalars");
  ctx->h_sc->timestep = h.timestep;
  ctx->h_sc->t = h.t;
  ctx->h_sc->prev_dt = h.prev_dt;
  ctx->h_sc->dt = h.dt;
  e = cudaMemcpyAsync(ctx->sc, ctx->h_sc, sizeof(DevScalars), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_check(ctx, e, "state scalars");
}

}  // extern "C"
