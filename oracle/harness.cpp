//------------------------------------------------------------------------------
// White-box oracle harness for the reference VAMPIRE CPU code.
//
// TEST INFRASTRUCTURE ONLY.  Linked against the reference's own object files
// (compiled by oracle/build_ref.py from the reference sources, unmodified).  It
// replaces the reference main() so that the system the reference builds, and
// the trajectory its own integrators produce, can be dumped bit-exactly:
//
//   * the reference start-up sequence of main() and sim::run() up to, not
//     including, the program switch (src/main/main.cpp:121-124,
//     src/simulate/sim.cpp:236-293);
//   * the CSR neighbour list and unrolled per-bond exchange list
//     (src/exchange/initialize.cpp:70-117, unroll_normalised.cpp:37-140,
//     dmi.cpp:46-221), material constants (initialise_variables.cpp:352-432),
//     reduced anisotropy constants (anisotropy/initialize.cpp:60-76);
//   * spins after N calls of sim::LLG_Heun() (LLGHeun.cpp:160-282) or
//     montecarlo::mc_step() (mc.cpp:29-127), each followed by the reference's
//     own time increment (sim.cpp:191-208, which updates the dipole field);
//   * the Gaussian thermal-noise stream the reference consumes in a step,
//     captured by saving the static MT19937 state, drawing 3N
//     mtrandom::gaussian() values in the x|y|z block order of
//     calculate_thermal_fields (fields.cpp:274-276) and restoring the state
//     (hdr/mtrand.hpp:62-64), so the reference then draws the same values;
//   * magnetisation and energy statistics (statistics/magnetization.cpp:134,
//     statistics/energy.cpp:141), torque statistics (utility/statistics.cpp:
//     221-325) and macrocell dipole fields (dipole/field.cpp).
//
// Output: raw little-endian arrays <name>.bin in --out, listed in manifest.txt
// as "<name> <dtype> <count>".
//------------------------------------------------------------------------------
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>
#include <chrono>
#include <cmath>

#include "atoms.hpp"
#include "anisotropy.hpp"
#include "cells.hpp"
#include "create.hpp"
#include "dipole.hpp"
#include "exchange.hpp"
#include "material.hpp"
#include "montecarlo.hpp"
#include "random.hpp"
#include "sim.hpp"
#include "stats.hpp"
#include "vio.hpp"
#include "vmpi.hpp"

#include "anisotropy/internal.hpp"
#include "exchange/internal.hpp"

namespace sim { void increment_time(); }
namespace stats { void system_torque(); }
namespace montecarlo { namespace cmc {
extern std::vector<std::vector<double> > polar_vector, polar_matrix;
} }

#ifdef VGPU_MC_HOOK
// Built as oracle/_ref/vampire-harness-b200 (reference objects compiled -DCUDA,
// the B200 vcuda:: backend, libvgpu.so): --gpu-mc runs the reference's
// start-up, then gpu::initialize(), and each Monte Carlo step through the
// gpu::mc_step hook a host adds in sim::integrate_serial (the two-line change
// INTEGRATION.md shows), i.e. vcuda::mc_step(), instead of
// montecarlo::mc_step.
#include "gpu.hpp"
namespace vcuda { void mc_step(); void cmc_step(); }
static bool g_gpu_mc = false;
#endif

// main.cpp owns this definition; the harness replaces main.cpp
namespace vmain { namespace internal { std::string input_file_name = "input"; } }

static std::string g_out = ".";
static std::ofstream g_manifest;

template <typename T>
static void dump(const std::string& name, const std::vector<T>& v, const char* dtype) {
   std::string path = g_out + "/" + name + ".bin";
   FILE* f = fopen(path.c_str(), "wb");
   if (!f) { std::cerr << "harness: cannot write " << path << std::endl; std::exit(2); }
   if (!v.empty()) fwrite(v.data(), sizeof(T), v.size(), f);
   fclose(f);
   g_manifest << name << " " << dtype << " " << v.size() << "\n";
   g_manifest.flush();
}
static void dumpd(const std::string& n, const std::vector<double>& v) { dump(n, v, "f8"); }
static void dumpi(const std::string& n, const std::vector<int>& v) { dump(n, v, "i4"); }

static std::vector<long> parse_list(const char* s) {
   std::vector<long> out;
   std::stringstream ss(s);
   std::string tok;
   while (std::getline(ss, tok, ',')) if (!tok.empty()) out.push_back(atol(tok.c_str()));
   return out;
}

static void dump_spins(const std::string& tag) {
   dumpd("sx_" + tag, atoms::x_spin_array);
   dumpd("sy_" + tag, atoms::y_spin_array);
   dumpd("sz_" + tag, atoms::z_spin_array);
}

static void dump_system() {
   const int n = atoms::num_atoms;
   std::vector<int> meta = {n, (int)atoms::total_num_neighbours, mp::num_materials,
                            (int)exchange::internal::exchange_type,
                            (int)anisotropy::internal::enable_uniaxial_second_order,
                            (int)anisotropy::internal::enable_cubic_fourth_order,
                            (int)dipole::activated, cells::num_cells,
                            (int)sim::hamiltonian_simulation_flags[3],
                            (int)sim::hamiltonian_simulation_flags[2]};
   dumpi("meta", meta);
   dumpi("nl_start", atoms::neighbour_list_start_index);
   dumpi("nl_end", atoms::neighbour_list_end_index);
   dumpi("nl", atoms::neighbour_list_array);
   dumpi("nl_type", atoms::neighbour_interaction_type_array);
   dumpi("type", atoms::type_array);
   dumpd("m_spin", atoms::m_spin_array);
   dumpd("cx", atoms::x_coord_array);
   dumpd("cy", atoms::y_coord_array);
   dumpd("cz", atoms::z_coord_array);
   // unrolled exchange list in its native form
   {
      std::vector<double> j;
      switch (exchange::internal::exchange_type) {
         case exchange::isotropic:
            for (auto& e : atoms::i_exchange_list) j.push_back(e.Jij);
            break;
         case exchange::vectorial:
            for (auto& e : atoms::v_exchange_list) for (int k = 0; k < 3; k++) j.push_back(e.Jij[k]);
            break;
         case exchange::tensorial:
            for (auto& e : atoms::t_exchange_list)
               for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) j.push_back(e.Jij[a][b]);
            break;
      }
      dumpd("jlist", j);
   }
   // per-material constants, 16 doubles per material
   std::vector<double> mat;
   for (int m = 0; m < mp::num_materials; m++) {
      const mp::materials_t& M = mp::material[m];
      double ku2 = anisotropy::internal::enable_uniaxial_second_order ? anisotropy::internal::ku2[m] : 0.0;
      double kc4 = (anisotropy::internal::enable_cubic_fourth_order ||
                    anisotropy::internal::enable_cubic_fourth_order_rotation) ? anisotropy::internal::kc4[m] : 0.0;
      double ex = 0, ey = 0, ez = 1;
      if (anisotropy::internal::ku_vector.size() > (size_t)m) {
         ex = anisotropy::internal::ku_vector[m].x;
         ey = anisotropy::internal::ku_vector[m].y;
         ez = anisotropy::internal::ku_vector[m].z;
      }
      double row[16] = {M.alpha, M.gamma_rel, M.mu_s_SI, M.one_oneplusalpha_sq, M.alpha_oneplusalpha_sq,
                        M.H_th_sigma, M.temperature_rescaling_alpha, M.temperature_rescaling_Tc,
                        ku2, ex, ey, ez, kc4, (double)M.non_magnetic, 0.0, 0.0};
      mat.insert(mat.end(), row, row + 16);
   }
   dumpd("materials", mat);
   // higher-order anisotropy: flags, per-material reduced constants [T] and the
   // normalised cubic basis, and the per-atom Neel tensors (anisotropy/internal.hpp)
   {
      namespace ai = anisotropy::internal;
      std::vector<int> fl = {(int)ai::enable_uniaxial_fourth_order, (int)ai::enable_uniaxial_sixth_order,
                             (int)ai::enable_cubic_sixth_order, (int)ai::enable_cubic_fourth_order_rotation,
                             (int)ai::enable_neel_anisotropy};
      dumpi("aniso_flags", fl);
      std::vector<double> ext;
      for (int m = 0; m < mp::num_materials; m++) {
         ext.push_back(ai::enable_uniaxial_fourth_order ? ai::ku4[m] : 0.0);
         ext.push_back(ai::enable_uniaxial_sixth_order ? ai::ku6[m] : 0.0);
         ext.push_back(ai::enable_cubic_sixth_order ? ai::kc6[m] : 0.0);
         for (int k = 0; k < 3; k++) ext.push_back(ai::mp[m].kc_vector1[k]);
         for (int k = 0; k < 3; k++) ext.push_back(ai::mp[m].kc_vector2[k]);
         for (int k = 0; k < 3; k++) ext.push_back(ai::mp[m].kc_vector3[k]);
      }
      dumpd("aniso_ext", ext);
      if (ai::enable_neel_anisotropy) dumpd("neel_tensor", ai::neel_tensor);
   }
   // biquadratic exchange: its own neighbour list and isotropic constants
   // (exchange/internal.hpp, exchange/biquadratic_fields.cpp)
   {
      namespace ei = exchange::internal;
      std::vector<int> bq = {(int)exchange::biquadratic, (int)ei::biquadratic_exchange_type};
      dumpi("bq_flag", bq);
      if (exchange::biquadratic) {
         dumpi("bq_start", ei::biquadratic_neighbour_list_start_index);
         dumpi("bq_end", ei::biquadratic_neighbour_list_end_index);
         dumpi("bq_nl", ei::biquadratic_neighbour_list_array);
         dumpi("bq_type", ei::biquadratic_neighbour_interaction_type_array);
         std::vector<double> j;
         for (auto& e : ei::bq_i_exchange_list) j.push_back(e.Jij);
         dumpd("bq_jlist", j);
      }
   }
   std::vector<double> simc = {mp::dt, mp::half_dt, mp::dt_SI, mp::gamma_SI, sim::temperature,
                               sim::H_applied, sim::H_vec[0], sim::H_vec[1], sim::H_vec[2]};
   dumpd("sim", simc);
   // statistics masks
   {
      std::vector<int> mask; std::vector<double> sat;
      stats::system_magnetization.get_mask(mask, sat);
      dumpi("mask_system", mask); dumpd("sat_system", sat);
      stats::material_magnetization.get_mask(mask, sat);
      dumpi("mask_material", mask); dumpd("sat_material", sat);
   }
   if (dipole::activated) {
      dumpi("cell_id", cells::atom_cell_id_array);
      dumpi("cell_natoms", cells::num_atoms_in_cell);
      dumpd("cell_volume", cells::volume_array);
      dumpd("cell_pos_mom", cells::pos_and_mom_array);
   }
}

// stats::system_torque and stats::max_torque (utility/statistics.cpp:221-325)
// at the current spins: the instantaneous system and per-material torque (the
// reference's sublattice sums, cleared first so one call's values remain)
// and the largest |S x H|.  Dumped as torque_<tag> = [T_x, T_y, T_z,
// T_x per material, T_y per material, T_z per material, max |S x H|].
static void dump_torque(const std::string& tag) {
   const int M = mp::num_materials;
   stats::num_atoms = atoms::num_atoms;
   stats::sublattice_mean_torque_x_array.assign(M, 0.0);
   stats::sublattice_mean_torque_y_array.assign(M, 0.0);
   stats::sublattice_mean_torque_z_array.assign(M, 0.0);
   stats::system_torque();
   std::vector<double> out(stats::total_system_torque, stats::total_system_torque + 3);
   for (int m = 0; m < M; m++) out.push_back(stats::sublattice_mean_torque_x_array[m]);
   for (int m = 0; m < M; m++) out.push_back(stats::sublattice_mean_torque_y_array[m]);
   for (int m = 0; m < M; m++) out.push_back(stats::sublattice_mean_torque_z_array[m]);
   out.push_back(stats::max_torque());
   dumpd("torque_" + tag, out);
}

static void dump_stats(const std::string& tag) {
   stats::update(atoms::x_spin_array, atoms::y_spin_array, atoms::z_spin_array,
                 atoms::m_spin_array, atoms::type_array, sim::temperature);
   std::vector<double> ms = stats::system_magnetization.get_magnetization();
   std::vector<double> mm = stats::material_magnetization.get_magnetization();
   dumpd("mag_system_" + tag, ms);
   dumpd("mag_material_" + tag, mm);
   std::vector<double> e;
   for (const std::vector<double>* v : {&stats::system_energy.get_total_energy(),
                                        &stats::system_energy.get_exchange_energy(),
                                        &stats::system_energy.get_anisotropy_energy(),
                                        &stats::system_energy.get_applied_field_energy(),
                                        &stats::system_energy.get_magnetostatic_energy()})
      e.insert(e.end(), v->begin(), v->end());
   dumpd("energy_system_" + tag, e);
   e.clear();
   for (const std::vector<double>* v : {&stats::material_energy.get_total_energy(),
                                        &stats::material_energy.get_exchange_energy(),
                                        &stats::material_energy.get_anisotropy_energy(),
                                        &stats::material_energy.get_applied_field_energy(),
                                        &stats::material_energy.get_magnetostatic_energy()})
      e.insert(e.end(), v->begin(), v->end());
   dumpd("energy_material_" + tag, e);
}

// the reference's derived statistics (susceptibility, specific heat, standard
// deviation), read back from their own output functions at 17 digits
static std::vector<double> parse_doubles(const std::string& text) {
   std::vector<double> v;
   std::istringstream ss(text);
   double x;
   while (ss >> x) v.push_back(x);
   return v;
}

static void dump_derived() {
   vout::custom_precision = true;
   vout::precision = 17;
   vout::fixed = false;
   const double T = sim::temperature;
   dumpd("sus_system", parse_doubles(stats::system_susceptibility.output_mean_susceptibility(T, false)));
   dumpd("sus_material", parse_doubles(stats::material_susceptibility.output_mean_susceptibility(T, false)));
   dumpd("spec_heat_system", parse_doubles(stats::system_specific_heat.output_mean_specific_heat(T, false)));
   dumpd("spec_heat_material", parse_doubles(stats::material_specific_heat.output_mean_specific_heat(T, false)));
   dumpd("std_material", parse_doubles(stats::material_standard_deviation.output_standard_deviation(false)));
}

static void dump_dipole(const std::string& tag) {
   if (!dipole::activated) return;
   dumpd("cmag_x_" + tag, cells::mag_array_x);
   dumpd("cmag_y_" + tag, cells::mag_array_y);
   dumpd("cmag_z_" + tag, cells::mag_array_z);
   dumpd("cfield_x_" + tag, dipole::cells_field_array_x);
   dumpd("cfield_y_" + tag, dipole::cells_field_array_y);
   dumpd("cfield_z_" + tag, dipole::cells_field_array_z);
   dumpd("chd_x_" + tag, dipole::cells_mu0Hd_field_array_x);
   dumpd("chd_y_" + tag, dipole::cells_mu0Hd_field_array_y);
   dumpd("chd_z_" + tag, dipole::cells_mu0Hd_field_array_z);
}

// one step of the selected integrator, as sim::integrate_serial dispatches it
// (src/simulate/sim.cpp:595-640)
static void one_step() {
   switch (sim::integrator) {
      case 1:
#ifdef VGPU_MC_HOOK
         if (g_gpu_mc) {
            vcuda::mc_step();
            break;
         }
#endif
         montecarlo::mc_step(atoms::x_spin_array, atoms::y_spin_array, atoms::z_spin_array, atoms::num_atoms,
                             atoms::type_array);
         break;
      case 2: sim::LLG_Midpoint(); break;
      case 4: montecarlo::cmc_mc_step(); break;
      case 3:
#ifdef VGPU_MC_HOOK
         if (g_gpu_mc) {
            vcuda::cmc_step();
            break;
         }
#endif
         montecarlo::cmc_step();
         break;
      default: sim::LLG_Heun(); break;
   }
}

int main(int argc, char* argv[]) {
   long steps = 0, warmup = 0, noise = 0, mag_every = 0, mag_start = 0, stats_every = 0;
   bool want_derived = false;
   std::vector<long> snaps, stat_snaps, torque_snaps;
   bool want_system = false, want_dipole = false, want_time = false;
   for (int i = 1; i < argc; i++) {
      std::string a = argv[i];
      auto next = [&]() -> const char* {
         if (i + 1 >= argc) { std::cerr << "harness: missing value for " << a << std::endl; std::exit(2); }
         return argv[++i];
      };
      if (a == "--out") g_out = next();
      else if (a == "--system") want_system = true;
      else if (a == "--steps") steps = atol(next());
      else if (a == "--warmup") warmup = atol(next());
      else if (a == "--snaps") snaps = parse_list(next());
      else if (a == "--noise") noise = atol(next());
      else if (a == "--stats") stat_snaps = parse_list(next());
      else if (a == "--torque") torque_snaps = parse_list(next());
      else if (a == "--mag-every") mag_every = atol(next());
      else if (a == "--mag-start") mag_start = atol(next());
      else if (a == "--dipole") want_dipole = true;
      else if (a == "--derived") want_derived = true;
      else if (a == "--stats-every") stats_every = atol(next());
      else if (a == "--time") want_time = true;
#ifdef VGPU_MC_HOOK
      else if (a == "--gpu-mc") g_gpu_mc = true;
#endif
      else { std::cerr << "harness: unknown option " << a << std::endl; return 2; }
   }
   g_manifest.open(g_out + "/manifest.txt");

   // reference start-up (main.cpp:56-124 without banner; sim.cpp:236-293)
   int one = 1; char* av[] = {argv[0], nullptr};
   vmpi::initialise(one, av);
   vout::zLogTsInit(std::string(argv[0]));
   stats::calculate_system_energy = true;
   stats::calculate_material_energy = true;
   if (want_derived) {
      stats::calculate_system_susceptibility = true;
      stats::calculate_material_susceptibility = true;
      stats::calculate_system_specific_heat = true;
      stats::calculate_material_specific_heat = true;
      stats::calculate_material_standard_deviation = true;
   }
   stats::calculate_system_magnetization = true;
   stats::calculate_material_magnetization = true;
   mp::initialise("input");
   cs::create();
   sim::initialize(mp::num_materials);
   montecarlo::initialize();
   anisotropy::initialize(atoms::num_atoms, atoms::type_array, mp::mu_s_array);
   mtrandom::grnd.seed(vmpi::parallel_rng_seed(mtrandom::integration_seed));
   {
      std::vector<bool> nonmag(mp::num_materials, false);
      for (int m = 0; m < mp::num_materials; m++) if (mp::material[m].non_magnetic == 2) nonmag[m] = true;
      stats::initialize(atoms::num_atoms, mp::num_materials, atoms::m_spin_array, atoms::type_array,
                        atoms::category_array, nonmag);
   }
   stats::update(atoms::x_spin_array, atoms::y_spin_array, atoms::z_spin_array, atoms::m_spin_array,
                 atoms::type_array, sim::temperature);
   dipole::initialize(cells::num_atoms_in_unit_cell, cells::num_cells, cells::num_local_cells,
                      cells::macro_cell_size, cells::local_cell_array, cells::num_atoms_in_cell,
                      cells::num_atoms_in_cell_global, cells::index_atoms_array, cells::volume_array,
                      cells::pos_and_mom_array, cells::atom_in_cell_coords_array_x,
                      cells::atom_in_cell_coords_array_y, cells::atom_in_cell_coords_array_z,
                      atoms::type_array, cells::atom_cell_id_array, atoms::x_coord_array,
                      atoms::y_coord_array, atoms::z_coord_array, atoms::x_spin_array,
                      atoms::y_spin_array, atoms::z_spin_array, atoms::m_spin_array, atoms::num_atoms);

#ifdef VGPU_MC_HOOK
   if (g_gpu_mc) {
      gpu::acceleration = true;
      gpu::initialize();
   }
#endif
   if (want_system) dump_system();
   dump_spins("0");
   if (want_dipole) dump_dipole("0");
   for (long s : stat_snaps) if (s == 0) dump_stats("0");
   for (long s : torque_snaps) if (s == 0) dump_torque("0");

   const int n = atoms::num_atoms;
   std::vector<double> mag_trace;  // per recorded step: mx, my, mz, |m| (system mask, bin 0), total E
   std::vector<double> mat_trace;  // per recorded step and material: m_x, m_y, m_z of that material
   // untimed warm-up steps (timing runs only; nothing is dumped for them)
   for (long w = 0; w < warmup; w++) {
      one_step();
      sim::increment_time();
   }
   const auto t0 = std::chrono::steady_clock::now();
   for (long step = 1; step <= steps; step++) {
      if (step <= noise) {
         std::vector<uint32_t> st(624);
         int32_t p = mtrandom::grnd.get_state(st);
         std::vector<double> xi(3 * (size_t)n);
         for (size_t k = 0; k < xi.size(); k++) xi[k] = mtrandom::gaussian();
         mtrandom::grnd.set_state(st, p);
         dumpd("xi_" + std::to_string(step), xi);
      }
      one_step();
      sim::increment_time();
#ifdef VGPU_MC_HOOK
      // the spins live on the device: bring them back where the host reads them
      if (g_gpu_mc && ((mag_every > 0 && step > mag_start && (step - mag_start) % mag_every == 0) ||
                       std::find(snaps.begin(), snaps.end(), step) != snaps.end()))
         gpu::config::synchronise();
#endif
      if (stats_every > 0 && step % stats_every == 0)
         stats::update(atoms::x_spin_array, atoms::y_spin_array, atoms::z_spin_array, atoms::m_spin_array,
                       atoms::type_array, sim::temperature);
      for (long s : snaps) if (s == step) dump_spins(std::to_string(step));
      for (long s : stat_snaps) if (s == step) dump_stats(std::to_string(step));
      for (long s : torque_snaps) if (s == step) dump_torque(std::to_string(step));
      if (want_dipole) for (long s : snaps) if (s == step) dump_dipole(std::to_string(step));
      if (mag_every > 0 && step > mag_start && (step - mag_start) % mag_every == 0) {
         double m[4] = {0, 0, 0, 0};
         for (int i = 0; i < n; i++) {
            m[0] += atoms::x_spin_array[i] * atoms::m_spin_array[i];
            m[1] += atoms::y_spin_array[i] * atoms::m_spin_array[i];
            m[2] += atoms::z_spin_array[i] * atoms::m_spin_array[i];
            m[3] += atoms::m_spin_array[i];
         }
         mag_trace.push_back(m[0] / m[3]);
         mag_trace.push_back(m[1] / m[3]);
         mag_trace.push_back(m[2] / m[3]);
         mag_trace.push_back(std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]) / m[3]);
         // per material: sum mu s / sum mu
         const int M = mp::num_materials;
         std::vector<double> mm(4 * M, 0.0);
         for (int i = 0; i < n; i++) {
            const int t = atoms::type_array[i];
            mm[4 * t + 0] += atoms::x_spin_array[i] * atoms::m_spin_array[i];
            mm[4 * t + 1] += atoms::y_spin_array[i] * atoms::m_spin_array[i];
            mm[4 * t + 2] += atoms::z_spin_array[i] * atoms::m_spin_array[i];
            mm[4 * t + 3] += atoms::m_spin_array[i];
         }
         for (int t = 0; t < M; t++)
            for (int q = 0; q < 3; q++) mat_trace.push_back(mm[4 * t + 3] > 0 ? mm[4 * t + q] / mm[4 * t + 3] : 0.0);
      }
   }
   const double loop_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
   if (want_time) std::cout << "HARNESS_LOOP_SECONDS " << loop_s << " ATOMS " << n << " STEPS " << steps << std::endl;
   if (!mag_trace.empty()) dumpd("mag_trace", mag_trace);
   if (!mat_trace.empty()) dumpd("mat_trace", mat_trace);
   if (want_derived) dump_derived();
#ifdef VGPU_MC_HOOK
   if (g_gpu_mc) gpu::finalize();
#endif
   if (sim::integrator == 4 && montecarlo::cmc::is_initialised) {
      // hybrid constrained Monte Carlo: every material's frame and the counters
      std::vector<double> fr;
      for (int m = 0; m < mp::num_materials; m++) {
         const auto& c = montecarlo::cmc::cmc_mat[m];
         for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) fr.push_back(c.ppolar_matrix[a][b]);
         for (int a = 0; a < 3; a++) fr.push_back(c.ppolar_vector[a]);
      }
      dumpd("cmc_frames", fr);
      std::vector<double> cc = {montecarlo::cmc::mc_total, montecarlo::cmc::mc_success,
                                montecarlo::cmc::energy_reject, montecarlo::cmc::sphere_reject};
      dumpd("cmc_counters", cc);
   }
   if (sim::integrator == 3 && montecarlo::cmc::is_initialised) {
      // constrained Monte Carlo: its frame (cmc.cpp polar_rot_matrix) and counters
      std::vector<double> fr;
      for (auto& row : montecarlo::cmc::polar_matrix) fr.insert(fr.end(), row.begin(), row.end());
      for (auto& row : montecarlo::cmc::polar_vector) fr.insert(fr.end(), row.begin(), row.end());
      dumpd("cmc_frame", fr);
      std::vector<double> cc = {montecarlo::cmc::mc_total, montecarlo::cmc::mc_success,
                                montecarlo::cmc::energy_reject, montecarlo::cmc::sphere_reject};
      dumpd("cmc_counters", cc);
   }
   std::vector<double> mc = {sim::mc_statistics_moves, sim::mc_statistics_reject};
   dumpd("mc_counters", mc);
   g_manifest.close();
   return 0;
}
