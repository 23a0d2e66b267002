//------------------------------------------------------------------------------
// vcuda:: backend of the VAMPIRE gpu:: facade, over libvgpu.so.
//
// The reference dispatches gpu::initialize / llg_heun / finalize /
// transfer_* / config::synchronise / stats::{update,get,reset}
// (src/gpu/*.cpp) to namespace vcuda (hdr/cuda.hpp:12-43) when built with
// -DCUDA; its own implementation is src/cuda/*.cu.  This file is a drop-in
// replacement for that directory: it is compiled together with the unmodified
// reference sources (-DCUDA) and reads the reference's globals exactly where
// src/cuda/initialize.cu did, marshals them into the plain descriptors of
// include/vgpu.h and calls the C ABI.  Nothing else in the reference changes.
//
// Behaviour kept from the reference:
//   * gpu::device selects the device (-1: current);
//   * gpu::cpu_stats (gpu:calculate-statistics-on-cpu, default true) copies
//     the spins to the host and runs the reference's own statistics classes,
//     as src/cuda/statistics.cu:30-49 does; otherwise statistics run on the
//     device (vgpu_stats_*), energies included;
//   * the macrocell and tensor dipole solvers run on the device: at
//     initialisation the cells:: arrays go to vgpu_dipole_setup, and
//     vgpu_llg_heun recomputes the field every dipole::update_rate steps
//     without leaving the device, so transfer_spin_positions_from_gpu_to_cpu
//     and transfer_dipole_fields_from_cpu_to_gpu -- the reference's
//     D2H / host update / H2D round trip around dipole::calculate_field
//     (dipole/field.cpp:43-87) -- have nothing to carry.  The atomistic
//     solver, or VGPU_DIPOLE=host in the environment, keeps the reference's
//     flow: the host computes the field and hands it over.
// Changed on purpose:
//   * finalize copies the spins back to the host first, so a checkpoint
//     written after the run (sim.cpp:521-524) holds the final spins;
//   * thermal noise is counter-based Philox keyed by
//     mtrandom::integration_seed; VGPU_PRECISION=fp64 in the environment
//     selects the FP64 build (bit-exact with sim::LLG_Heun).
//------------------------------------------------------------------------------
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "atoms.hpp"
#include "anisotropy.hpp"
#include "cuda.hpp"
#include "dipole.hpp"
#include "errors.hpp"
#include "exchange.hpp"
#include "gpu.hpp"
#include "material.hpp"
#include "montecarlo.hpp"
#include "random.hpp"
#include "sim.hpp"
#include "stats.hpp"
#include "vio.hpp"

#include "anisotropy/internal.hpp"
#include "cells.hpp"
#include "dipole/internal.hpp"
#include "exchange/internal.hpp"

#include "vgpu.h"

namespace {

vgpu_handle g_h = nullptr;
bool g_cpu_stats = true;
vgpu_sim_params g_last;
bool g_have_last = false;
// device statistics masks: system, material, height, material-height
int32_t g_mask_id[4] = {-1, -1, -1, -1};
int32_t g_mask_size[4] = {0, 0, 0, 0};
bool g_dipole_device = false;  // the device dipole solver holds the field

void fail(int rc, const char* what) {
   if (rc == VGPU_OK) return;
   char buf[1024];
   vgpu_last_error(g_h, buf, sizeof buf);
   std::cerr << "Error: GPU " << what << " failed (" << rc << "): " << buf << std::endl;
   zlog << zTs() << "Error: GPU " << what << " failed (" << rc << "): " << buf << std::endl;
   err::vexit();
}

vgpu_sim_params current_params() {
   vgpu_sim_params p;
   std::memset(&p, 0, sizeof p);
   p.dt = mp::dt;
   p.temperature = sim::temperature;
   p.H_applied = sim::H_applied;
   p.H_vec[0] = sim::H_vec[0];
   p.H_vec[1] = sim::H_vec[1];
   p.H_vec[2] = sim::H_vec[2];
   p.thermal_enabled = sim::hamiltonian_simulation_flags[3];
   p.applied_enabled = sim::hamiltonian_simulation_flags[2];
   p.local_temperature = sim::local_temperature;
   p.local_applied_field = sim::local_applied_field;
   return p;
}

// the simulate programs change temperature and field between steps
void sync_params() {
   const vgpu_sim_params p = current_params();
   if (g_have_last && std::memcmp(&p, &g_last, sizeof p) == 0) return;
   fail(vgpu_set_params(g_h, &p), "set_params");
   g_last = p;
   g_have_last = true;
}

void add_mask(int k, ::stats::magnetization_statistic_t& st, bool enabled) {
   if (!enabled || !st.is_initialized()) return;
   std::vector<int> mask;
   std::vector<double> sat;
   st.get_mask(mask, sat);
   if ((int)mask.size() != ::atoms::num_atoms) return;
   g_mask_size[k] = (int32_t)sat.size();
   fail(vgpu_stats_add_mask(g_h, mask.data(), g_mask_size[k], &g_mask_id[k]), "stats mask");
}

void get_mask(int k, ::stats::magnetization_statistic_t& st) {
   if (g_mask_id[k] < 0) return;
   std::vector<double> m(4 * g_mask_size[k]), mean(4 * g_mask_size[k]);
   int64_t counter = 0;
   fail(vgpu_stats_get_magnetization(g_h, g_mask_id[k], m.data(), mean.data(), &counter), "stats get");
   // the averages are kept on the device (src/cuda/statistics.cu:270-277)
   st.reset_magnetization_averages();
   st.set_magnetization(m, mean, (long)counter);
}

void spins_to_host() {
   fail(vgpu_get_spins(g_h, ::atoms::x_spin_array.data(), ::atoms::y_spin_array.data(),
                       ::atoms::z_spin_array.data()), "spin download");
}

}  // namespace

namespace vcuda {

bool initialize(bool cpu_stats) {
   g_cpu_stats = cpu_stats;
   const char* prec_env = std::getenv("VGPU_PRECISION");
   const int prec = (prec_env && std::string(prec_env) == "fp64") ? VGPU_PREC_FP64 : VGPU_PREC_FP32;
   if (vgpu_create(gpu::device, prec, &g_h) != VGPU_OK) {
      char buf[1024];
      vgpu_last_error(nullptr, buf, sizeof buf);
      std::cerr << "Error: unable to initialise the B200 backend: " << buf << std::endl;
      zlog << zTs() << "Error: unable to initialise the B200 backend: " << buf << std::endl;
      return false;
   }
   zlog << zTs() << "B200 backend " << vgpu_version() << " on device " << gpu::device << std::endl;

   // materials (initialise_variables.cpp:423-432, anisotropy/initialize.cpp:60-76)
   const int M = mp::num_materials;
   std::vector<vgpu_material> mats(M);
   for (int m = 0; m < M; ++m) {
      vgpu_material& q = mats[m];
      std::memset(&q, 0, sizeof q);
      const mp::materials_t& src = mp::material[m];
      q.alpha = src.alpha;
      q.gamma_rel = src.gamma_rel;
      q.mu_s_SI = src.mu_s_SI;
      q.one_oneplusalpha_sq = src.one_oneplusalpha_sq;
      q.alpha_oneplusalpha_sq = src.alpha_oneplusalpha_sq;
      q.H_th_sigma = src.H_th_sigma;
      q.temperature_rescaling_alpha = src.temperature_rescaling_alpha;
      q.temperature_rescaling_Tc = src.temperature_rescaling_Tc;
      if (anisotropy::internal::enable_uniaxial_second_order) q.ku2 = anisotropy::internal::ku2[m];
      if ((int)anisotropy::internal::ku_vector.size() > m) {
         q.ku_vector[0] = anisotropy::internal::ku_vector[m].x;
         q.ku_vector[1] = anisotropy::internal::ku_vector[m].y;
         q.ku_vector[2] = anisotropy::internal::ku_vector[m].z;
      } else {
         q.ku_vector[2] = 1.0;
      }
      if (anisotropy::internal::enable_cubic_fourth_order || anisotropy::internal::enable_cubic_fourth_order_rotation)
         q.kc4 = anisotropy::internal::kc4[m];
      q.temperature = src.temperature;
      if (src.applied_field_unit_vector.size() >= 3)
         for (int k = 0; k < 3; ++k) q.applied_field[k] = src.applied_field_strength * src.applied_field_unit_vector[k];
      q.non_magnetic = src.non_magnetic;
   }

   // system: CSR and unrolled exchange list (exchange/initialize.cpp:70-117)
   vgpu_system_desc d;
   std::memset(&d, 0, sizeof d);
   d.num_atoms = ::atoms::num_atoms;
   d.num_materials = M;
   d.exchange_type = (int32_t)exchange::internal::exchange_type;
   d.uniaxial_enabled = anisotropy::internal::enable_uniaxial_second_order;
   d.cubic_enabled = anisotropy::internal::enable_cubic_fourth_order;
   d.num_bonds = (int64_t)::atoms::neighbour_list_array.size();
   d.nl_start = ::atoms::neighbour_list_start_index.data();
   d.nl_end = ::atoms::neighbour_list_end_index.data();
   d.nl = ::atoms::neighbour_list_array.data();
   d.nl_type = ::atoms::neighbour_interaction_type_array.data();
   std::vector<double> jl;
   switch (exchange::internal::exchange_type) {
      case exchange::isotropic:
         for (auto& e : ::atoms::i_exchange_list) jl.push_back(e.Jij);
         break;
      case exchange::vectorial:
         for (auto& e : ::atoms::v_exchange_list) for (int k = 0; k < 3; ++k) jl.push_back(e.Jij[k]);
         break;
      default:
         for (auto& e : ::atoms::t_exchange_list)
            for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) jl.push_back(e.Jij[a][b]);
         break;
   }
   const int w = d.exchange_type == VGPU_EXCH_ISOTROPIC ? 1 : d.exchange_type == VGPU_EXCH_VECTORIAL ? 3 : 9;
   d.num_exchange = (int64_t)jl.size() / w;
   d.jlist = jl.data();
   d.type = ::atoms::type_array.data();
   d.materials = mats.data();
   d.sx = ::atoms::x_spin_array.data();
   d.sy = ::atoms::y_spin_array.data();
   d.sz = ::atoms::z_spin_array.data();
   fail(vgpu_upload_system(g_h, &d), "system upload");
   // higher-order anisotropy (anisotropy/internal.hpp), as anisotropy::fields evaluates it
   {
      namespace ai = anisotropy::internal;
      if (ai::enable_lattice_anisotropy) {
         std::cerr << "Error: lattice anisotropy is not evaluated by the B200 backend" << std::endl;
         zlog << zTs() << "Error: lattice anisotropy is not evaluated by the B200 backend" << std::endl;
         err::vexit();
      }
      vgpu_anisotropy_ext x;
      std::memset(&x, 0, sizeof x);
      x.uniaxial_fourth = ai::enable_uniaxial_fourth_order;
      x.uniaxial_sixth = ai::enable_uniaxial_sixth_order;
      x.cubic_sixth = ai::enable_cubic_sixth_order;
      x.cubic_rotation = ai::enable_cubic_fourth_order_rotation;
      x.neel = ai::enable_neel_anisotropy;
      std::vector<double> kcb;
      if (x.uniaxial_fourth) x.ku4 = ai::ku4.data();
      if (x.uniaxial_sixth) x.ku6 = ai::ku6.data();
      if (x.cubic_sixth) x.kc6 = ai::kc6.data();
      if (x.cubic_rotation) {
         for (int m = 0; m < M; ++m) {
            for (int k = 0; k < 3; ++k) kcb.push_back(ai::mp[m].kc_vector1[k]);
            for (int k = 0; k < 3; ++k) kcb.push_back(ai::mp[m].kc_vector2[k]);
            for (int k = 0; k < 3; ++k) kcb.push_back(ai::mp[m].kc_vector3[k]);
         }
         x.kc_basis = kcb.data();
      }
      if (x.neel) x.neel_tensor = ai::neel_tensor.data();
      if (x.uniaxial_fourth || x.uniaxial_sixth || x.cubic_sixth || x.cubic_rotation || x.neel)
         fail(vgpu_set_anisotropy_ext(g_h, &x), "higher-order anisotropy");
   }
   // biquadratic exchange (exchange/internal.hpp): isotropic constants only, as
   // exchange::single_spin_biquadratic_energy evaluates them
   if (exchange::biquadratic) {
      namespace ei = exchange::internal;
      if (ei::biquadratic_exchange_type != exchange::isotropic) {
         std::cerr << "Error: only isotropic biquadratic exchange is evaluated by the B200 backend" << std::endl;
         err::vexit();
      }
      std::vector<double> bj;
      for (auto& e : ei::bq_i_exchange_list) bj.push_back(e.Jij);
      vgpu_biquadratic_desc b;
      std::memset(&b, 0, sizeof b);
      b.num_bonds = (int64_t)ei::biquadratic_neighbour_list_array.size();
      b.nl_start = ei::biquadratic_neighbour_list_start_index.data();
      b.nl_end = ei::biquadratic_neighbour_list_end_index.data();
      b.nl = ei::biquadratic_neighbour_list_array.data();
      b.nl_type = ei::biquadratic_neighbour_interaction_type_array.data();
      b.num_exchange = (int64_t)bj.size();
      b.jlist = bj.data();
      fail(vgpu_set_biquadratic(g_h, &b), "biquadratic exchange");
   }
   sync_params();
   fail(vgpu_set_noise(g_h, VGPU_NOISE_PHILOX, (uint64_t)(uint32_t)mtrandom::integration_seed), "noise");
   fail(vgpu_set_step(g_h, sim::time), "step counter");

   if (!g_cpu_stats) {
      add_mask(0, ::stats::system_magnetization, ::stats::calculate_system_magnetization);
      add_mask(1, ::stats::material_magnetization, ::stats::calculate_material_magnetization);
      add_mask(2, ::stats::height_magnetization, ::stats::calculate_height_magnetization);
      add_mask(3, ::stats::material_height_magnetization, ::stats::calculate_material_height_magnetization);
   }
   if (dipole::activated) {
      const char* where = std::getenv("VGPU_DIPOLE");
      const bool host = (where && std::string(where) == "host") ||
                        dipole::internal::solver == dipole::internal::atomistic;
      if (host) {
         // per-atom fields computed on the host at start-up (dipole::initialize)
         transfer_dipole_fields_from_cpu_to_gpu();
      } else {
         // the device solver: macrocells as cells::initialize built them
         // (cells/initialize.cpp:189-265), field computed now from the spins
         vgpu_dipole_desc dd;
         std::memset(&dd, 0, sizeof dd);
         dd.num_cells = cells::num_cells;
         dd.solver = dipole::internal::solver == dipole::internal::tensor ? VGPU_DIPOLE_TENSOR : VGPU_DIPOLE_MACROCELL;
         dd.update_rate = dipole::update_rate;
         dd.macro_cell_size = cells::macro_cell_size;
         dd.cutoff = dipole::cutoff;
         dd.atom_cell = cells::atom_cell_id_array.data();
         dd.cell_pos_mom = cells::pos_and_mom_array.data();
         dd.cell_volume = cells::volume_array.data();
         dd.cell_natoms = cells::num_atoms_in_cell.data();
         dd.atom_x = ::atoms::x_coord_array.data();
         dd.atom_y = ::atoms::y_coord_array.data();
         dd.atom_z = ::atoms::z_coord_array.data();
         fail(vgpu_dipole_setup(g_h, &dd), "dipole setup");
         g_dipole_device = true;
         zlog << zTs() << "B200 backend: macrocell dipole field on the device (" << cells::num_cells
              << " cells, update every " << dipole::update_rate << " steps)" << std::endl;
      }
   }
   return true;
}

void llg_heun() {
   sync_params();
   fail(vgpu_llg_heun(g_h, 1), "llg_heun");
}

void stats_update() { stats::update(); }

// LLG-Midpoint step on the GPU (sim::LLG_Midpoint, src/simulate/LLGMidpoint.cpp);
// hdr/cuda.hpp has no such entry: a host that adds gpu::llg_midpoint()
// forwards it here from the llg-midpoint case of sim::integrate_serial.
void llg_midpoint();
void llg_midpoint() {
   sync_params();
   fail(vgpu_llg_midpoint(g_h, 1), "llg_midpoint");
}

// Metropolis sweep on the GPU: N angle-move trials, one per atom, in colour
// order (the reference's montecarlo::mc_step, src/montecarlo/mc.cpp:29-127,
// makes N random-site trials on the host).  hdr/cuda.hpp has no such entry;
// a host that adds gpu::mc_step() forwards it here.  Angle moves only: other
// montecarlo::algorithm values stay on the host.
void mc_step();
void mc_step() {
   static bool setup = false;
   if (!setup) {
      int32_t nc = 0;
      fail(vgpu_mc_setup(g_h, nullptr, &nc), "mc setup");
      fail(vgpu_mc_set_sweep(g_h, sim::time), "mc sweep counter");
      setup = true;
   }
   sync_params();
   fail(vgpu_mc_sweep(g_h, 1), "mc sweep");
   double moves = 0.0, rejects = 0.0;
   fail(vgpu_mc_counters(g_h, &moves, &rejects), "mc counters");
   sim::mc_statistics_moves = moves;
   sim::mc_statistics_reject = rejects;
}

// Constrained Monte Carlo step on the GPU (montecarlo::cmc_step,
// src/montecarlo/cmc.cpp:282-490): about N pair moves; the first call sets
// the constraint (sim::constraint_phi, sim::constraint_theta) and, unless a
// checkpoint was loaded, turns the spins along it as CMCinit does.  hdr/cuda.hpp
// has no such entry; a host that adds gpu::cmc_step() forwards it here.
void cmc_step();
void cmc_step() {
   static bool setup = false;
   if (!setup) {
      fail(vgpu_cmc_setup(g_h, sim::constraint_phi, sim::constraint_theta, sim::checkpoint_loaded_flag ? 0 : 1),
           "cmc setup");
      setup = true;
   }
   sync_params();
   fail(vgpu_cmc_sweep(g_h, 1), "cmc step");
   double c[4];
   fail(vgpu_cmc_get(g_h, nullptr, c), "cmc counters");
   montecarlo::cmc::mc_total = c[0];
   montecarlo::cmc::mc_success = c[1];
   montecarlo::cmc::energy_reject = c[2];
   montecarlo::cmc::sphere_reject = c[3];
   montecarlo::cmc::is_initialised = true;
}

void finalize() {
   if (!g_h) return;
   spins_to_host();
   vgpu_destroy(g_h);
   g_h = nullptr;
   g_dipole_device = false;
}

// called by dipole::calculate_field around its host update; with the device
// solver the field is already current on the device, so nothing crosses
void transfer_spin_positions_from_gpu_to_cpu() {
   if (g_h && !g_dipole_device) spins_to_host();
}

void transfer_dipole_fields_from_cpu_to_gpu() {
   if (!g_h || g_dipole_device) return;
   fail(vgpu_set_dipole_field(g_h, dipole::atom_dipolar_field_array_x.data(), dipole::atom_dipolar_field_array_y.data(),
                              dipole::atom_dipolar_field_array_z.data(), dipole::atom_mu0demag_field_array_x.data(),
                              dipole::atom_mu0demag_field_array_y.data(), dipole::atom_mu0demag_field_array_z.data()),
        "dipole field upload");
}

namespace config {
void synchronise() {
   if (g_h) spins_to_host();
}
}  // namespace config

namespace stats {

void update() {
   // sim::run calls stats::update once before gpu::initialize (sim.cpp:264 vs
   // :296): the host spins are current then, so the host classes do it
   if (g_cpu_stats || !g_h) {
      // reference behaviour (src/cuda/statistics.cu:32-49)
      if (g_h) spins_to_host();
      if (::stats::calculate_system_magnetization)
         ::stats::system_magnetization.calculate_magnetization(::atoms::x_spin_array, ::atoms::y_spin_array, ::atoms::z_spin_array, ::atoms::m_spin_array);
      if (::stats::calculate_material_magnetization)
         ::stats::material_magnetization.calculate_magnetization(::atoms::x_spin_array, ::atoms::y_spin_array, ::atoms::z_spin_array, ::atoms::m_spin_array);
      if (::stats::calculate_height_magnetization)
         ::stats::height_magnetization.calculate_magnetization(::atoms::x_spin_array, ::atoms::y_spin_array, ::atoms::z_spin_array, ::atoms::m_spin_array);
      if (::stats::calculate_material_height_magnetization)
         ::stats::material_height_magnetization.calculate_magnetization(::atoms::x_spin_array, ::atoms::y_spin_array, ::atoms::z_spin_array, ::atoms::m_spin_array);
      return;
   }
   fail(vgpu_stats_update(g_h, 1), "stats update");
}

void get() {
   if (g_cpu_stats || !g_h) return;
   get_mask(0, ::stats::system_magnetization);
   get_mask(1, ::stats::material_magnetization);
   get_mask(2, ::stats::height_magnetization);
   get_mask(3, ::stats::material_height_magnetization);
}

void reset() {
   if (g_cpu_stats || !g_h) {
      if (::stats::calculate_system_magnetization) ::stats::system_magnetization.reset_magnetization_averages();
      if (::stats::calculate_material_magnetization) ::stats::material_magnetization.reset_magnetization_averages();
      if (::stats::calculate_height_magnetization) ::stats::height_magnetization.reset_magnetization_averages();
      if (::stats::calculate_material_height_magnetization)
         ::stats::material_height_magnetization.reset_magnetization_averages();
      return;
   }
   fail(vgpu_stats_reset(g_h), "stats reset");
}

}  // namespace stats

}  // namespace vcuda
