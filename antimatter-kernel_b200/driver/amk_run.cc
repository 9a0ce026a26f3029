// amk_run: the reference application's main loop (antimatter-kernel.cc:41-216)
// on libamk, with the state resident on the GPU.
//
//   amk_run [params.json] [output_dir] [--checkpoint PATH --checkpoint-every N]
//           [--resume PATH] [--vtk-every N]
//
// Reads the reference's params.json keys, validates them as the reference
// does, creates the reference's initial cloud (bit-identical generators),
// and steps Coulomb -> Lorentz + cooling -> annihilation. Energies follow
// the reference's schedule and format: a time-centred evaluation at step 0,
// then every num_steps / 100 steps (and the last step), each evaluation
// also run on the step before a logged step so that the time-centring pairs
// consecutive steps; lines "step N  KE=... PE_trap=... PE_coulomb=...
// TOTAL=... J" on stdout and the same CSV columns in
// <output_dir>/energy_analysis_data.csv; drift relative to the trap depth
// e |U|. With coulomb forces disabled the Coulomb energy column is 0, as in
// the reference. Final positions are printed as the reference does; set
// AMK_RUN_NO_POSITIONS=1 to skip them for large clouds.
//
// In place of BioDynaMo's backup/restore and visualisation export:
// --checkpoint PATH --checkpoint-every N writes a checkpoint every N steps
// (amk_checkpoint_save) plus PATH.driver holding the step-0 energies the
// drift is measured from; --resume PATH continues such a run up to the
// params file's num_steps (same CSV rows and lines as the uninterrupted run
// from the resumed step on, appended to an existing CSV); --vtk-every N writes output_dir/particles_<step>.vtu
// (binary VTK XML of the live particles) at step 0 and every N steps, and
// output_dir/particles.pvd listing them.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "amk.h"

namespace {

int die(const char* what) {
  std::cerr << "amk_run: " << what << ": " << amk_last_error() << std::endl;
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  const auto start = std::chrono::high_resolution_clock::now();
  std::vector<std::string> pos;
  std::string ckpt_path, resume_path;
  long ckpt_every = 0, vtk_every = 0;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if ((a == "--checkpoint" || a == "--resume" || a == "--checkpoint-every" || a == "--vtk-every") && i + 1 < argc) {
      const std::string v = argv[++i];
      if (a == "--checkpoint") ckpt_path = v;
      else if (a == "--resume") resume_path = v;
      else if (a == "--checkpoint-every") ckpt_every = std::atol(v.c_str());
      else vtk_every = std::atol(v.c_str());
    } else {
      pos.push_back(a);
    }
  }
  const std::string params_path = pos.size() > 0 ? pos[0] : "params.json";
  const std::string out_dir = pos.size() > 1 ? pos[1] : "output";
  amk_params p;
  amk_params_default(&p);
  if (amk_params_load_json(params_path.c_str(), &p) != AMK_OK) return die("params");
  if (amk_params_validate(&p, 1) != AMK_OK) return die("params");
  const char* dev = std::getenv("AMK_DEVICE");
  amk_ctx* ctx = nullptr;
  if (amk_create(&p, dev ? std::atoi(dev) : 0, &ctx) != AMK_OK) return die("context");
  long first_step = 1;
  amk_energy_out e0{};
  bool have_e0 = false;
  if (!resume_path.empty()) {
    // the checkpoint's parameters and state; the run length is this params file's
    const long run_steps = p.num_steps;
    if (amk_checkpoint_load(ctx, resume_path.c_str()) != AMK_OK) return die("resume");
    if (amk_get_params(ctx, &p) != AMK_OK) return die("resume");
    p.num_steps = run_steps;
    if (amk_set_params(ctx, &p) != AMK_OK) return die("resume");
    first_step = amk_step_count(ctx) + 1;
    std::ifstream side(resume_path + ".driver");
    if (!(side >> e0.kinetic >> e0.trap_potential >> e0.coulomb_potential >> e0.total >> e0.num_active)) {
      std::cerr << "amk_run: missing " << resume_path << ".driver (the step-0 energies)" << std::endl;
      return 1;
    }
    have_e0 = true;
  } else if (amk_init_particles(ctx) != AMK_OK) {
    return die("initial particles");
  }
  std::vector<std::string> vtk_files;
  std::vector<double> vtk_times;
  auto export_vtk = [&](long step) -> bool {
    const std::string name = "particles_" + std::to_string(step) + ".vtu";
    if (amk_export_vtk(ctx, (out_dir + "/" + name).c_str(), 1) != AMK_OK) return false;
    vtk_files.push_back(name);
    vtk_times.push_back(static_cast<double>(step) * p.dt);
    return true;
  };

  const long num_steps = p.num_steps;
  const long log_interval = num_steps >= 100 ? num_steps / 100 : 1;
  auto evaluate = [&](amk_energy_out* e) -> bool {
    if (amk_energy(ctx, 1, e) != AMK_OK) return false;
    if (!p.coulomb_forces_enabled) {
      e->coulomb_potential = 0.0;
      e->total = e->kinetic + e->trap_potential;
    }
    return true;
  };

  const std::string csv_path = out_dir + "/energy_analysis_data.csv";
  std::ofstream csv(csv_path, have_e0 ? std::ios::app : std::ios::trunc);
  if (!csv.is_open())
    std::cerr << "WARNING: could not open '" << csv_path << "' for writing -- energy CSV will not be saved this run."
              << std::endl;
  else if (!have_e0)
    csv << "step,kinetic_energy_J,trap_potential_energy_J,potential_energy_J,total_energy_J,num_active_particles,"
           "fractional_drift,absolute_drift_J\n";

  if (!have_e0) {
    if (!evaluate(&e0)) return die("energy");
    std::cout << "\nstep 0  KE=" << e0.kinetic << " PE_trap=" << e0.trap_potential << " PE_coulomb="
              << e0.coulomb_potential << " TOTAL=" << e0.total << " J" << std::endl;
    if (csv.is_open())
      csv << 0 << "," << e0.kinetic << "," << e0.trap_potential << "," << e0.coulomb_potential << "," << e0.total
          << "," << e0.num_active << "," << 0.0 << "," << 0.0 << "\n";
    if (vtk_every > 0 && !export_vtk(0)) return die("vtk export");
  }
  double scale = 1.602176634e-19 * std::fabs(p.trap_voltage);
  if (scale <= 0.0) scale = std::fabs(e0.total);
  if (scale <= 0.0) scale = 1.0;

  for (long step = first_step; step <= num_steps; ++step) {
    if (amk_step(ctx, 1) != AMK_OK) return die("step");
    if (vtk_every > 0 && step % vtk_every == 0 && !export_vtk(step)) return die("vtk export");
    const bool log_step = (step % log_interval == 0) || (step == num_steps);
    const bool need = log_step || ((step + 1) % log_interval == 0) || (step + 1 == num_steps);
    if (need) {
      amk_energy_out e;
      if (!evaluate(&e)) return die("energy");
      if (log_step) {
        const double absolute = e.total - e0.total;
        const double fractional = absolute / scale;
        std::cout << "step " << step << "  KE=" << e.kinetic << " PE_trap=" << e.trap_potential
                  << " PE_coulomb=" << e.coulomb_potential << " TOTAL=" << e.total << " J"
                  << "  (drift: " << absolute << " J, " << fractional << " of trap depth)" << std::endl;
        if (csv.is_open())
          csv << step << "," << e.kinetic << "," << e.trap_potential << "," << e.coulomb_potential << ","
              << e.total << "," << e.num_active << "," << fractional << "," << absolute << "\n";
      }
    }
    // after this step's energy evaluation, so the time-centring history of
    // a resumed run is the uninterrupted run's
    if (!ckpt_path.empty() && ckpt_every > 0 && step % ckpt_every == 0) {
      if (amk_checkpoint_save(ctx, ckpt_path.c_str()) != AMK_OK) return die("checkpoint");
      std::ofstream side(ckpt_path + ".driver");
      side.precision(17);
      side << e0.kinetic << " " << e0.trap_potential << " " << e0.coulomb_potential << " " << e0.total << " "
           << e0.num_active << "\n";
      if (csv.is_open()) csv.flush();
    }
  }
  if (csv.is_open()) {
    csv.close();
    std::cout << "Energy analysis written to: " << csv_path << std::endl;
  }
  if (!vtk_files.empty()) {
    std::vector<const char*> names;
    for (const auto& f : vtk_files) names.push_back(f.c_str());
    if (amk_write_pvd((out_dir + "/particles.pvd").c_str(), static_cast<long>(names.size()), names.data(),
                      vtk_times.data()) != AMK_OK)
      return die("vtk collection");
  }
  if (!std::getenv("AMK_RUN_NO_POSITIONS")) {
    const long n = amk_num_particles(ctx);
    std::vector<double> x(n), y(n), z(n), vx(n), vy(n), vz(n);
    std::vector<uint8_t> alive(n);
    if (amk_get_particles(ctx, x.data(), y.data(), z.data(), vx.data(), vy.data(), vz.data(), alive.data()) != AMK_OK)
      return die("particles");
    for (long i = 0; i < n; ++i)
      std::cout << "final position: (" << x[i] << ", " << y[i] << ", " << z[i] << ")" << std::endl;
  }
  amk_destroy(ctx);
  const std::chrono::duration<double> took = std::chrono::high_resolution_clock::now() - start;
  std::cout << "Simulation completed successfully!" << std::endl;
  std::cout << "Time taken " << took.count() << "s" << std::endl;
  return 0;
}
