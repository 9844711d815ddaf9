// imex_run: the time-marching driver of the reference's main() (main.cpp:334-595) over the
// C ABI, with the state on the GPU for the whole run.
//
//   imex_run <config file> <initial state file> <output directory>
//
// The config file holds "name = value" lines with the reference's names (config.hpp:43-125:
// formula, magfield, recon, caltimestep, CFL, GMREStol, p_floor, ...; enumerators by name or
// ordinal), the domain x_0 x_1 y_0 y_1, time_stop, RKs, and the driver's own keys:
//   plot_interval  VTK every k steps besides step 0 and the end (0: those two only)
//   max_steps      stop after this many steps even before time_stop (0: no cap)
//   name           prefix of the VTK files (plt_<name>_<step>.vtk)
// The initial state is a state file (imex_save_state_file; the Python problems write them).
// Per step the reference's console lines are printed ("[timestep, dt, time] = ...,
// Divergence Error: ...", "DIAG ts=..." and the four "[CT-DIAG]" lines of its EMF
// decomposition, main.cpp:562-594), and after the run the output directory holds
// the VTK files, the histories RK_div_error.dat, RK_B_inf.dat, RK_dt_comp.dat, the field
// files RK_*.dat and final_state.bin.
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "imex_b200.h"

namespace {

struct Field {
  const char* name;
  bool is_int;
  size_t offset;
};
#define FI(f) {#f, true, offsetof(imex_config, f)}
#define FD(f) {#f, false, offsetof(imex_config, f)}
const Field kFields[] = {
    FI(caltimestep), FI(formula),  FI(magfield), FI(add_pvisc), FI(flux_diss), FI(GLF), FI(add_bvisc),
    FI(U_update), FI(vortex_test), FI(RKs), FD(CFL), FI(recon), FI(reconstate), FI(x_bc), FI(y_bc),
    FI(PressureSolver), FI(Energy_Modify), FD(GMREStol), FD(shock_kappa1), FI(floor_on), FD(p_floor),
    FD(Mbig_fac), FD(theta), FI(Pnewton_max), FD(Pnewton_tol), FI(eos_type), FD(gamma_plasma), FD(m_alfa),
    FD(m_b), FD(m_R), FD(m_cv), FD(x_0), FD(x_1), FD(y_0), FD(y_1), FD(time_stop), FD(fixed_dt),
    FI(gmres_restart), FI(gmres_max_restarts), FI(precision), FD(mixed_inner_tol), FI(mixed_max_refine),
    FI(mixed_solves)};
#undef FI
#undef FD

// enumerators of config.hpp:27-41,118 by name
const std::map<std::string, int> kEnums = {
    {"EnergyFormula", IMEX_EnergyFormula}, {"PressureFormula", IMEX_PressureFormula},
    {"StaggerCT", IMEX_StaggerCT}, {"UnStaggerCT", IMEX_UnStaggerCT}, {"PotentialA", IMEX_PotentialA},
    {"NoDivFree", IMEX_NoDivFree}, {"NoRecon", IMEX_NoRecon}, {"Minmod", IMEX_Minmod}, {"VanLeer", IMEX_VanLeer},
    {"ENO3", IMEX_ENO3}, {"WENO5", IMEX_WENO5}, {"PrimState", IMEX_PrimState}, {"ConsState", IMEX_ConsState},
    {"Fullydt", IMEX_Fullydt}, {"Alfvendt", IMEX_Alfvendt}, {"IMEXdt", IMEX_IMEXdt},
    {"x_Transmissive", IMEX_x_Transmissive}, {"x_Reflective", IMEX_x_Reflective}, {"x_Periodic", IMEX_x_Periodic},
    {"x_Dirichlet", IMEX_x_Dirichlet}, {"y_Transmissive", IMEX_y_Transmissive},
    {"y_Reflective", IMEX_y_Reflective}, {"y_Periodic", IMEX_y_Periodic}, {"y_Dirichlet", IMEX_y_Dirichlet},
    {"y_JetInflow", IMEX_y_JetInflow}, {"MaterialSpeedp", IMEX_MaterialSpeedp},
    {"AlfvenSpeedp", IMEX_AlfvenSpeedp}, {"Noaddvisp", IMEX_Noaddvisp}, {"ConservationofU", IMEX_ConservationofU},
    {"DefinitionofU", IMEX_DefinitionofU}, {"Local_Diss", IMEX_Local_Diss}, {"Global_Diss", IMEX_Global_Diss},
    {"no_correction", IMEX_no_correction}, {"once_correction", IMEX_once_correction},
    {"all_correction", IMEX_all_correction}, {"IDEAL_GAS", IMEX_IDEAL_GAS}, {"REDLICH_KWONG", IMEX_REDLICH_KWONG},
    {"fp64", IMEX_PRECISION_FP64}, {"mixed", IMEX_PRECISION_MIXED}};

std::string trim(const std::string& s) {
  const size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

struct Run {
  imex_config cfg;
  int nx = 0, ny = 0;
  int plot_interval = 0;
  long max_steps = 0;
  std::string name = "run";
};

bool parse(const char* path, Run& r, std::string& err) {
  std::ifstream in(path);
  if (!in) return err = std::string("cannot read ") + path, false;
  imex_config_default(&r.cfg);
  std::string line;
  int ln = 0;
  while (std::getline(in, line)) {
    ++ln;
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    line = trim(line);
    if (line.empty()) continue;
    const size_t eq = line.find('=');
    if (eq == std::string::npos) return err = "line " + std::to_string(ln) + ": expected name = value", false;
    const std::string key = trim(line.substr(0, eq)), val = trim(line.substr(eq + 1));
    if (key == "nx") { r.nx = std::atoi(val.c_str()); continue; }
    if (key == "ny") { r.ny = std::atoi(val.c_str()); continue; }
    if (key == "plot_interval") { r.plot_interval = std::atoi(val.c_str()); continue; }
    if (key == "max_steps") { r.max_steps = std::atol(val.c_str()); continue; }
    if (key == "name") { r.name = val; continue; }
    const Field* f = nullptr;
    for (const Field& q : kFields)
      if (key == q.name) f = &q;
    if (!f) return err = "line " + std::to_string(ln) + ": unknown key '" + key + "'", false;
    char* base = reinterpret_cast<char*>(&r.cfg) + f->offset;
    if (f->is_int) {
      auto it = kEnums.find(val);
      int v = it != kEnums.end() ? it->second : std::atoi(val.c_str());
      std::memcpy(base, &v, sizeof(int));
    } else {
      double v = std::strtod(val.c_str(), nullptr);
      std::memcpy(base, &v, sizeof(double));
    }
  }
  if (r.nx < 1 || r.ny < 1) return err = "nx and ny are required", false;
  return true;
}

int fail(imex_ctx* ctx, imex_status s, const char* what) {
  std::fprintf(stderr, "imex_run: %s: %s (%s)\n", what, imex_status_string(s), ctx ? imex_last_error(ctx) : "");
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: %s <config file> <initial state file> <output directory>\n", argv[0]);
    return 2;
  }
  Run r;
  std::string err;
  if (!parse(argv[1], r, err)) {
    std::fprintf(stderr, "imex_run: %s: %s\n", argv[1], err.c_str());
    return 2;
  }
  const std::string out = argv[3];
  imex_ctx* ctx = nullptr;
  imex_status s = imex_create(&r.cfg, r.nx, r.ny, &ctx);
  if (s != IMEX_OK) return fail(ctx, s, "imex_create");
  if ((s = imex_load_state_file(ctx, argv[2])) != IMEX_OK) return fail(ctx, s, "initial state");
  auto vtk = [&](int step) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "_%d.vtk", step);
    const std::string path = out + "/plt_" + r.name + buf;
    return imex_write_vtk(ctx, path.c_str(), step);
  };
  imex_diagnostics_t d{};
  if ((s = imex_diagnostics(ctx, &d)) != IMEX_OK) return fail(ctx, s, "diagnostics");
  if ((s = vtk(d.timestep)) != IMEX_OK) return fail(ctx, s, "VTK");
  std::vector<int> steps;
  std::vector<double> div, binf, dtc;
  long n = 0;
  while (d.t < r.cfg.time_stop && (r.max_steps <= 0 || n < r.max_steps)) {
    double dt = 0.0;
    if ((s = imex_step(ctx, &dt)) != IMEX_OK) return fail(ctx, s, "imex_step");
    ++n;
    if ((s = imex_diagnostics(ctx, &d)) != IMEX_OK) return fail(ctx, s, "diagnostics");
    std::printf("[timestep, dt, time] = %d %.17g %.17g, Divergence Error: %.17g\n", d.timestep, dt, d.t, d.div_error);
    std::printf("DIAG ts=%d t=%.17g emin=%.17g at(%.17g,%.17g) mass=%.17g intE=%.17g magE_max=%.17g\n", d.timestep,
                d.t, d.emin, d.emin_x, d.emin_y, d.mass, d.intE, d.magE_max);
    double ct[16];
    if ((s = imex_ct_emf_diagnostics(ctx, ct)) != IMEX_OK) return fail(ctx, s, "CT EMF diagnostics");
    static const char* parts[4] = {"central", "rusanov", "tilde", "TOTAL"};
    for (int c = 0; c < 4; ++c)
      std::printf("[CT-DIAG] %-8s  Ez: L2=%.3e max=%.3e | dB/dt: L2=%.3e max=%.3e\n", parts[c], ct[4 * c],
                  ct[4 * c + 1], ct[4 * c + 2], ct[4 * c + 3]);
    steps.push_back(d.timestep);
    div.push_back(d.div_error);
    binf.push_back(d.B_inf);
    dtc.push_back(d.dt_comp);
    if (r.plot_interval > 0 && d.timestep % r.plot_interval == 0 && (s = vtk(d.timestep)) != IMEX_OK)
      return fail(ctx, s, "VTK");
  }
  if (!(r.plot_interval > 0 && d.timestep % r.plot_interval == 0) && (s = vtk(d.timestep)) != IMEX_OK)
    return fail(ctx, s, "VTK");
  const int ns = (int)steps.size();
  if (imex_history_write_host((out + "/RK_div_error.dat").c_str(), ns, steps.data(), div.data()) != IMEX_OK ||
      imex_history_write_host((out + "/RK_B_inf.dat").c_str(), ns, steps.data(), binf.data()) != IMEX_OK ||
      imex_history_write_host((out + "/RK_dt_comp.dat").c_str(), ns, steps.data(), dtc.data()) != IMEX_OK)
    return fail(ctx, IMEX_ERR_INVALID, "histories");
  if ((s = imex_write_fields_dat(ctx, out.c_str())) != IMEX_OK) return fail(ctx, s, "field files");
  if ((s = imex_save_state_file(ctx, (out + "/final_state.bin").c_str())) != IMEX_OK) return fail(ctx, s, "state");
  imex_destroy(ctx);
  return 0;
}
