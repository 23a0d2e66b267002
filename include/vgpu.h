/*
 * vgpu.h -- C ABI of libvgpu.so, the B200 (sm_100a) spin-update library.
 *
 * This is the boundary a VAMPIRE host binds to.  It replaces the body of the
 * reference's CUDA backend (namespace vcuda, hdr/cuda.hpp:12-43, implemented
 * in src/cuda/*.cu), which the reference's gpu:: facade (hdr/gpu.hpp:13-58,
 * src/gpu/*.cpp) dispatches to.  The reference host reads its physics from
 * globals (atoms::, mp::material, sim::, dipole::, cells::, stats::); the
 * vcuda shim (vampire_b200/host/vcuda_b200.cpp) marshals those globals into
 * the plain descriptors below.  No torch or CUDA types appear here: plain
 * pointers to host memory and sizes only.  The library copies on upload and on
 * download; the caller owns every host buffer.
 *
 * Every function returns an int status: VGPU_OK (0) or a negative VGPU_ERR_*.
 * vgpu_last_error() gives the message of the last failure on a handle (or the
 * last failure of a handle-less call when h is NULL).  Calls on one handle
 * must be serialised by the caller (the reference is single-threaded);
 * different handles are independent.  No call blocks forever: device-side
 * waits are bounded and surface as VGPU_ERR_TIMEOUT.
 */
#ifndef VGPU_H_
#define VGPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VGPU_OK            0
#define VGPU_ERR_ARG      -1  /* invalid argument or descriptor              */
#define VGPU_ERR_CUDA     -2  /* CUDA runtime error                          */
#define VGPU_ERR_OOM      -3  /* device allocation failed                    */
#define VGPU_ERR_TIMEOUT  -4  /* a bounded device-side wait gave up          */
#define VGPU_ERR_NAN      -5  /* non-finite spin detected                    */
#define VGPU_ERR_STATE    -6  /* call out of order (e.g. no system uploaded) */

/* exchange representation of the per-bond list, as exchange::internal::exchange_type
 * (hdr/exchange_types.hpp): isotropic = 0, vectorial = 1, tensorial = 2 */
#define VGPU_EXCH_ISOTROPIC 0
#define VGPU_EXCH_VECTORIAL 1
#define VGPU_EXCH_TENSORIAL 2

/* arithmetic of the device state */
#define VGPU_PREC_FP32 0      /* production: FP32 state, FP64 reductions       */
#define VGPU_PREC_FP64 1      /* debug/oracle build: FP64 everywhere           */

/* source of the Gaussian thermal noise */
#define VGPU_NOISE_PHILOX 0   /* counter-based Philox4x32-10, in-register      */
#define VGPU_NOISE_REPLAY 1   /* host-supplied 3N values (x|y|z blocks), for    *
                               * replaying the reference mtrandom stream        */

typedef struct vgpu_ctx* vgpu_handle;

/* Per-material constants, as the reference derives them in
 * set_derived_parameters (src/main/initialise_variables.cpp:423-432) and
 * anisotropy::initialize (src/anisotropy/initialize.cpp:60-76). */
typedef struct {
   double alpha;                   /* Gilbert damping                                   */
   double gamma_rel;               /* relative gyromagnetic ratio                       */
   double mu_s_SI;                 /* moment [J/T]                                      */
   double one_oneplusalpha_sq;     /* -gamma_rel/(1+alpha^2)                            */
   double alpha_oneplusalpha_sq;   /* alpha * one_oneplusalpha_sq                       */
   double H_th_sigma;              /* sqrt(2 alpha kB/(mu_s gamma_rel dt))              */
   double temperature_rescaling_alpha;
   double temperature_rescaling_Tc;
   double ku2;                     /* reduced 2nd-order uniaxial constant Ku/mu_s [T]   */
   double ku_vector[3];            /* uniaxial easy axis (unit vector)                  */
   double kc4;                     /* reduced 4th-order cubic constant Kc/mu_s [T]      */
   double temperature;             /* material temperature (used if local_temperature)  */
   double applied_field[3];        /* material local applied field [T]                  */
   int32_t non_magnetic;           /* non-zero: excluded from cell moments              */
   int32_t pad_;
} vgpu_material;

/* One spin system: the reference's CSR neighbour list and unrolled exchange
 * list (src/exchange/initialize.cpp:70-117, unroll_normalised.cpp:37-140). */
typedef struct {
   int32_t num_atoms;
   int32_t num_materials;
   int32_t exchange_type;          /* VGPU_EXCH_*                                       */
   int32_t uniaxial_enabled;       /* anisotropy::internal::enable_uniaxial_second_order */
   int32_t cubic_enabled;          /* anisotropy::internal::enable_cubic_fourth_order    */
   int32_t pad_;
   int64_t num_bonds;              /* atoms::total_num_neighbours                       */
   const int32_t* nl_start;        /* [num_atoms] atoms::neighbour_list_start_index      */
   const int32_t* nl_end;          /* [num_atoms] atoms::neighbour_list_end_index (incl.)*/
   const int32_t* nl;              /* [num_bonds] atoms::neighbour_list_array            */
   const int32_t* nl_type;         /* [num_bonds] interaction id, or NULL = bond index   */
   int64_t num_exchange;           /* entries in jlist                                   */
   const double* jlist;            /* [num_exchange * {1,3,9}] J in Tesla (i/v/t list;   *
                                    * tensors row-major Jij[a][b])                        */
   const int32_t* type;            /* [num_atoms] material id (atoms::type_array)        */
   const vgpu_material* materials; /* [num_materials]                                    */
   const double* sx;               /* [num_atoms] initial spin (unit vectors)            */
   const double* sy;
   const double* sz;
} vgpu_system_desc;

/* Simulation parameters (namespace sim / mp in the reference). */
typedef struct {
   double dt;                      /* reduced time step mp::dt = dt_SI * gamma_SI       */
   double temperature;             /* sim::temperature [K]                              */
   double H_applied;               /* sim::H_applied [T]                                */
   double H_vec[3];                /* sim::H_vec                                        */
   int32_t thermal_enabled;        /* sim::hamiltonian_simulation_flags[3]              */
   int32_t applied_enabled;        /* sim::hamiltonian_simulation_flags[2]              */
   int32_t local_temperature;      /* sim::local_temperature                            */
   int32_t local_applied_field;    /* sim::local_applied_field                          */
} vgpu_sim_params;

/* ---- life cycle --------------------------------------------------------- */

/* Create a context on CUDA device `device` (-1: current device) with its own
 * stream.  precision is VGPU_PREC_FP32 or VGPU_PREC_FP64.
 * Replaces vcuda::initialize device selection (src/cuda/initialize.cu:84-105). */
int vgpu_create(int device, int precision, vgpu_handle* out);

/* Free every device buffer of the handle.  Replaces vcuda::finalize
 * (src/cuda/finalize.cu). */
int vgpu_destroy(vgpu_handle h);

/* Copy the message of the last error into buf (NUL-terminated). */
int vgpu_last_error(vgpu_handle h, char* buf, size_t n);

/* Library version string, e.g. "vgpu 0.1 sm_100a". */
const char* vgpu_version(void);

/* ---- system upload ------------------------------------------------------ */

/* Upload atoms, CSR, exchange list, materials and spins.  Re-uploading
 * replaces the system.  Validates the CSR on the host first (monotone,
 * 0 <= neighbour < num_atoms) and returns VGPU_ERR_ARG with a message if it
 * is malformed.  Replaces vcuda::initialize's marshalling of atoms, fields,
 * materials and topology (src/cuda/initialize.cu:398-515). */
int vgpu_upload_system(vgpu_handle h, const vgpu_system_desc* desc);

/* Higher-order anisotropy beyond the descriptor's second-order uniaxial and
 * fourth-order cubic terms, as the reference's anisotropy module evaluates
 * them (src/anisotropy/fields.cpp:42-63, energy.cpp:27-36):
 * uniaxial_fourth_order.cpp, uniaxial_sixth_order.cpp (along the material's
 * ku_vector), cubic_fourth_order_rotation.cpp (kc4 of vgpu_material in the
 * basis e1, e2, e3; replaces the plain cubic term, so cubic_enabled = 0),
 * cubic_sixth_order.cpp and neel.cpp (per-atom surface tensors built by
 * initialize_neel.cpp).  Constants are the reduced ones of
 * anisotropy::internal (K / mu_s, Tesla).  Call after vgpu_upload_system;
 * a new upload clears them.  Replaces the part of vcuda::initialize that
 * never reached the device (src/cuda/spin_fields.cu:95-152 has no such terms). */
typedef struct {
   int32_t uniaxial_fourth;        /* enable_uniaxial_fourth_order                      */
   int32_t uniaxial_sixth;         /* enable_uniaxial_sixth_order                       */
   int32_t cubic_sixth;            /* enable_cubic_sixth_order                          */
   int32_t cubic_rotation;         /* enable_cubic_fourth_order_rotation                */
   int32_t neel;                   /* enable_neel_anisotropy                            */
   int32_t pad_;
   const double* ku4;              /* [num_materials] or NULL when off                  */
   const double* ku6;              /* [num_materials] or NULL when off                  */
   const double* kc6;              /* [num_materials] or NULL when off                  */
   const double* kc_basis;         /* [num_materials][9] e1, e2, e3 (unit, orthogonal)  */
   const double* neel_tensor;      /* [num_atoms][9] row-major 3x3 [T], or NULL         */
} vgpu_anisotropy_ext;
int vgpu_set_anisotropy_ext(vgpu_handle h, const vgpu_anisotropy_ext* a);

/* Biquadratic exchange (exchange::biquadratic; material biquadratic-exchange
 * or unit-cell biquadratic interactions): H_i += sum_j 2 J_bq (s_i.s_j) s_j
 * over its own CSR list (src/exchange/biquadratic_fields.cpp:60-76), energy
 * -sum_j J_bq (s_i.s_j)^2 counted with the exchange energy
 * (biquadratic_energy.cpp, statistics/energy.cpp:165-173).  Isotropic
 * constants in Tesla (bq_i_exchange_list), as the reference evaluates them.
 * Call after vgpu_upload_system. */
typedef struct {
   int64_t num_bonds;
   const int32_t* nl_start;        /* [num_atoms] biquadratic_neighbour_list_start_index */
   const int32_t* nl_end;          /* [num_atoms] ..._end_index (inclusive)              */
   const int32_t* nl;              /* [num_bonds] biquadratic_neighbour_list_array       */
   const int32_t* nl_type;         /* [num_bonds] interaction id, or NULL = bond index   */
   int64_t num_exchange;           /* entries in jlist                                   */
   const double* jlist;            /* [num_exchange] J_bq [T]                            */
} vgpu_biquadratic_desc;
int vgpu_set_biquadratic(vgpu_handle h, const vgpu_biquadratic_desc* b);

/* Host-only check of a descriptor (no device needed): CSR rows inside
 * [0, num_bonds), neighbours and interaction ids in range, materials in
 * range, finite spins.  VGPU_ERR_ARG / VGPU_ERR_NAN with a message for
 * vgpu_last_error(NULL, ...).  vgpu_upload_system runs the same check. */
int vgpu_validate_system(const vgpu_system_desc* desc);

/* Set time step, temperature and applied field; may be called between steps. */
int vgpu_set_params(vgpu_handle h, const vgpu_sim_params* p);

/* ---- spin access -------------------------------------------------------- */

/* Overwrite the device spins from host arrays of num_atoms doubles. */
int vgpu_set_spins(vgpu_handle h, const double* sx, const double* sy, const double* sz);

/* Copy the device spins to host arrays (num_atoms doubles each).  Replaces
 * vcuda::transfer_spin_positions_from_gpu_to_cpu and
 * vcuda::config::synchronise (src/cuda/transfer.cu, src/cuda/config.cu:25-34). */
int vgpu_get_spins(vgpu_handle h, double* sx, double* sy, double* sz);

/* ---- LLG-Heun ----------------------------------------------------------- */

/* Noise source.  VGPU_NOISE_PHILOX with a 64-bit seed (the default, seed 0),
 * or VGPU_NOISE_REPLAY: the next step uses the 3*num_atoms values last given
 * to vgpu_set_noise_replay (x block, then y, then z: the order of
 * calculate_thermal_fields, src/simulate/fields.cpp:274-276). */
int vgpu_set_noise(vgpu_handle h, int mode, uint64_t seed);
int vgpu_set_noise_replay(vgpu_handle h, const double* xi);

/* Options.  VGPU_OPT_STORE_INCREMENT: 1 = the predictor stores f(s0) for the
 * corrector (3 extra arrays, +24 B per spin-step), 0 = the corrector recovers
 * f(s0) dt = s'|s0|^2/(s'.s0) - s0 from the two states it reads anyway;
 * -1 (default) = store in FP64 (bit-exact with the reference), recover in FP32. */
#define VGPU_OPT_STORE_INCREMENT 1
/* VGPU_OPT_STAGED_RECORDS (FP32 systems with DMI/vector bond records): 1 = the
 * fused passes bring each tile's bond records into shared memory with one bulk
 * copy per tile, 0 = every thread loads its own records, -1 (default) = staged
 * when a tile's buffers fit in 200 KB of shared memory.  Same results bit for
 * bit either way.  VGPU_OPT_STAGE_SLICES: 2, 4 or 8 slices of 32 atoms per
 * tile; VGPU_OPT_STAGE_BUFFERS: 1 (one tile per block) or 2 (persistent
 * blocks, next tile's copy overlapping this one); -1 (default) = the measured
 * best for the record layout: 4 slices, 1 buffer with 16-byte records; 2
 * slices, 2 buffers with compact records.  A copy that does not complete
 * within a bounded wait fails the step with VGPU_ERR_TIMEOUT. */
#define VGPU_OPT_STAGED_RECORDS 2
#define VGPU_OPT_STAGE_SLICES 3
#define VGPU_OPT_STAGE_BUFFERS 4
/* VGPU_OPT_DIPOLE_FFT (read by vgpu_dipole_setup): 1 or -1 (default) = the
 * far-field cell sum by FP64 FFT convolution when every occupied cell centre
 * lies on one regular grid (falls back to the direct sum otherwise), 0 =
 * always the direct all-pairs sum. */
#define VGPU_OPT_DIPOLE_FFT 5
/* VGPU_OPT_STAGE_WAIT_TEST: 1 = staged passes wait for 16 bytes more than each
 * tile's copy delivers, so their bounded wait (1 s) runs out and the step
 * fails with VGPU_ERR_TIMEOUT (test of the timeout path; the handle stays
 * usable after setting it back to 0). */
#define VGPU_OPT_STAGE_WAIT_TEST 6
/* VGPU_OPT_COMPACT_RECORDS (FP32 systems with DMI bond records): 1 or -1
 * (default) = when the system has at most 512 distinct bond couplings (and
 * enough index bits above the neighbour index), the fused passes read one
 * 4-byte word per bond (neighbour | coupling index) and take the coupling from
 * a dictionary instead of a 16-byte record; 0 = always the 16-byte records.
 * Same results bit for bit either way (the same coupling values). */
#define VGPU_OPT_COMPACT_RECORDS 7
/* VGPU_OPT_WINDOW_STAGING (staged passes over compact records, one buffer):
 * 1 = each tile also stages its "window" -- the contiguous atom ranges holding
 * every neighbour of its atoms, planned on the host at the first pass -- into
 * shared memory with bulk copies, and gathers neighbour spins from there (used
 * when every tile's window fits in 4096 atoms and 256 ranges); 0 or -1
 * (default) = gathers through L1/L2 (measured faster on B200).  Same results
 * bit for bit. */
#define VGPU_OPT_WINDOW_STAGING 8
/* VGPU_OPT_PROFILE_EVERY: with vgpu_profile on, time the launches of one step
 * in `value` (>= 1; default 1 = every launch).  The events recorded around a
 * timed launch delay the stream by a few microseconds, so sampling keeps a
 * profiled run close to an unprofiled one. */
#define VGPU_OPT_PROFILE_EVERY 9
/* VGPU_OPT_STAGE_WARPS (staged passes over compact records, no window
 * staging): 2 or 4 = per-warp pipelined passes with that many warps per
 * persistent block, every warp walking its own one-slice tiles with two
 * buffers and no block-wide barrier; 0 or -1 (default) = the tile passes.
 * The results are the same bit for bit. */
#define VGPU_OPT_STAGE_WARPS 10
/* Bond-record layout the next FP32 pass reads: *layout = VGPU_RECORDS_WINDOW
 * (compact words with window staging), VGPU_RECORDS_COMPACT,
 * VGPU_RECORDS_WIDE (16-byte records) or VGPU_RECORDS_NONE (formats without
 * packed records, and FP64); *dict_entries (optional) = coupling dictionary
 * size (0 when no compact records were built).  Plans the window if the next
 * pass would. */
#define VGPU_RECORDS_NONE 0
#define VGPU_RECORDS_WIDE 1
#define VGPU_RECORDS_COMPACT 2
#define VGPU_RECORDS_WINDOW 3
int vgpu_record_layout(vgpu_handle h, int32_t* layout, int32_t* dict_entries);
/* Per-bond exchange format chosen at upload for the reference's unrolled
 * exchange list (src/exchange/unroll.cpp, unroll_normalised.cpp): the
 * coupling is read from a material-pair table when it is a function of the
 * two materials (VGPU_EXCH_ISO_TAB / VEC_TAB / DMI_TAB: diagonal table plus
 * the antisymmetric part per bond), else stored per bond (ISO_BOND: scalar,
 * VEC_BOND: diagonal, TENSOR_BOND: full 3x3). */
#define VGPU_EXCH_ISO_TAB 0
#define VGPU_EXCH_ISO_BOND 1
#define VGPU_EXCH_VEC_TAB 2
#define VGPU_EXCH_VEC_BOND 3
#define VGPU_EXCH_DMI_TAB 4
#define VGPU_EXCH_TENSOR_BOND 5
int vgpu_exchange_format(vgpu_handle h, int32_t* fmt);
int vgpu_set_option(vgpu_handle h, int option, int value);

/* Step counter that keys the Philox stream (counter = (atom, step)).  Resume
 * from a checkpoint by restoring it. */
int vgpu_set_step(vgpu_handle h, uint64_t step);
int vgpu_get_step(vgpu_handle h, uint64_t* step);

/* Advance n_steps stochastic Heun steps (src/simulate/LLGHeun.cpp:160-282):
 * one fused predictor and one fused corrector launch per step.  Replaces
 * vcuda::llg_heun (src/cuda/llg_heun.cu:32-42,121-208). */
int vgpu_llg_heun(vgpu_handle h, uint64_t n_steps);

/* ---- spatial shards (one process per GPU, halo exchange between passes) ---
 * No reference counterpart in the gpu:: interface; they carry the reference's
 * MPI decomposition (core/boundary/halo atoms, src/simulate/LLGHeun-mpi.cpp:
 * 62-64, halo refresh src/mpi/mpi_comms.cpp:45-143) onto one GPU per rank. */

/* One fused pass: VGPU_PASS_PREDICTOR (s' from s) or VGPU_PASS_CORRECTOR (s
 * from s and s'; completes the step: counter and dipole cadence).
 * vgpu_llg_heun(h, 1) is the predictor followed by the corrector.  The
 * external field (thermal, applied, macrocell dipole) belongs to the step, as
 * in the reference, which computes it once per step: with the record-staged
 * passes the corrector uses the field the predictor computed, so parameters
 * changed between the two passes of a step take effect at the next step. */
#define VGPU_PASS_PREDICTOR 0
#define VGPU_PASS_CORRECTOR 1
int vgpu_llg_pass(vgpu_handle h, int pass);

/* One pass over part of the updated atoms, first_atom .. end_atom - 1
 * (first_atom a multiple of 32, end_atom at most the owned count): a shard
 * runs its core atoms while the halo exchange of the pass's input state is in
 * flight, then its boundary atoms -- the reference's split around
 * mpi_init_halo_swap / mpi_complete_halo_swap (src/mpi/LLGHeun-mpi.cpp:61-140).
 * The corrector range that ends at the last owned atom completes the step
 * (step counter, dipole cadence), so the ranges of a corrector pass run in
 * ascending order of their end.  Not with window staging. */
int vgpu_llg_pass_range(vgpu_handle h, int pass, int32_t first_atom, int32_t end_atom);

/* The uploaded system is a shard: atoms 0..n_owned-1 are owned and updated
 * by the passes (and summed by the statistics); the rest are halo copies of
 * other ranks' atoms that the host refreshes between passes.  noise_base is
 * added to the atom index in the Philox counter: the global index of owned
 * atom 0 when the owned atoms are one contiguous global range, so that the
 * shard draws the noise of the whole system.  Call it before vgpu_mc_setup
 * and vgpu_dipole_setup_shard. */
int vgpu_set_owned(vgpu_handle h, int32_t n_owned, int64_t noise_base);

/* Halo transfers, queued on the handle's stream (vgpu_get_stream) with
 * DEVICE buffers of the handle's precision: pack gathers state `which`
 * (VGPU_STATE_SPIN = s, VGPU_STATE_PREDICTOR = s') at the count local indices
 * idx[] into out[3*count] (x block, y, z); unpack writes in[3*count] into
 * atoms first..first+count-1. */
#define VGPU_STATE_SPIN 0
#define VGPU_STATE_PREDICTOR 1
int vgpu_halo_pack(vgpu_handle h, int which, const int32_t* idx, int32_t count, void* out);
int vgpu_halo_unpack(vgpu_handle h, int which, int32_t first, int32_t count, const void* in);
/* The same on another stream of the handle's device (a cudaStream_t as
 * void*), so that a shard's exchange runs beside its core-range pass; the
 * caller orders them with events: the pack after the pass that wrote the
 * state, the boundary-range pass after the unpack. */
int vgpu_halo_pack_on(vgpu_handle h, int which, const int32_t* idx, int32_t count, void* out, void* stream);
int vgpu_halo_unpack_on(vgpu_handle h, int which, int32_t first, int32_t count, const void* in, void* stream);

/* Advance n_steps of the LLG-Midpoint integrator (sim::LLG_Midpoint,
 * src/simulate/LLGMidpoint.cpp:48-150; sim:integrator=llg-midpoint): the
 * same two fused passes per step as vgpu_llg_heun -- the first writes the
 * midpoint M = (S + R S)/2 (Cayley rotation with F = H + alpha S x H), the
 * second rotates S by F(M, H(M)) -- with the external field, thermal noise
 * included, shared by both halves.  No renormalisation, as the reference.
 * The reference runs this integrator on the host only. */
int vgpu_llg_midpoint(vgpu_handle h, uint64_t n_steps);

/* Write the 3*num_atoms Gaussians (x|y|z blocks) that the Philox stream
 * gives the thermal field at step `step` -- the values the fused kernels
 * regenerate in-register.  For tests and for replaying a run elsewhere. */
int vgpu_thermal_noise(vgpu_handle h, uint64_t step, double* xi);

/* Total (spin + external) field the predictor sees at the current spins, in
 * Tesla, with thermal noise excluded (debug/parity aid). */
int vgpu_get_fields(vgpu_handle h, double* hx, double* hy, double* hz);

/* ---- macrocell dipole field ---------------------------------------------- */

#define VGPU_DIPOLE_MACROCELL 0   /* bare point dipoles, self term 0 (dipole/macrocell.cpp)   */
#define VGPU_DIPOLE_TENSOR    1   /* atomistic tensors within cutoff (dipole/tensor.cpp)      */

/* Macrocells as the reference's cells:: module builds them
 * (src/cells/initialize.cpp:189-265). */
typedef struct {
   int32_t num_cells;              /* cells::num_cells                                   */
   int32_t solver;                 /* VGPU_DIPOLE_*  (dipole::internal::solver)          */
   int32_t update_rate;            /* steps between updates (dipole::update_rate); 0: never */
   int32_t pad_;
   double macro_cell_size;         /* cells::macro_cell_size [Angstrom]                  */
   double cutoff;                  /* dipole::cutoff [macrocell sizes]                   */
   const int32_t* atom_cell;       /* [num_atoms] cells::atom_cell_id_array              */
   const double* cell_pos_mom;     /* [4*num_cells] cells::pos_and_mom_array             */
   const double* cell_volume;      /* [num_cells] cells::volume_array [Angstrom^3]       */
   const int32_t* cell_natoms;     /* [num_cells] cells::num_atoms_in_cell               */
   const double* atom_x;           /* [num_atoms] atomic coordinates [Angstrom]          */
   const double* atom_y;           /*   (tensor solver only; else may be NULL)           */
   const double* atom_z;
} vgpu_dipole_desc;

/* Enable the device dipole solver and compute the field at the current spins
 * (dipole::initialize, src/dipole/initialize.cpp:143).  vgpu_llg_heun then
 * recomputes it every update_rate steps (dipole::calculate_field,
 * src/dipole/field.cpp:43-87) without leaving the device: cell moments
 * (cells::mag, src/cells/mag.cpp:35-77) and cell fields
 * (dipole::internal::update_field, src/dipole/update.cpp:37-105) replace the
 * reference's D2H-CPU-H2D round trip and its O(Nc^2) dense tensors. */
int vgpu_dipole_setup(vgpu_handle h, const vgpu_dipole_desc* desc);

/* Recompute cell moments and fields now (on a shard: the partial moments,
 * as at the dipole cadence). */
int vgpu_dipole_update(vgpu_handle h);

/* The device dipole solver on a shard (vgpu_set_owned first).  `whole`
 * describes the whole system of n_global atoms: the cell arrays as for
 * vgpu_dipole_setup (cells of the whole system, the reference's cells::
 * arrays after their MPI_Allreduce, src/cells/initialize.cpp:237-242), and
 * atom_cell (and for the tensor solver atom_x/y/z) of every global atom;
 * global_type[n_global] are the material ids, local[i] the global id of the
 * shard's atom i.  The near tensors are built from all global atoms (the
 * reference exchanges the atoms of neighbouring cells between ranks,
 * src/dipole/tensor.cpp:63-135).
 *
 * At setup and at every update (the cadence in the corrector pass, or
 * vgpu_dipole_update) the shard sums its OWNED atoms into the cell moments
 * and stops: the caller adds the moment buffer (vgpu_dipole_moment_buffer)
 * over all ranks in place -- the reference's MPI_Allreduce of
 * cells::mag_array (src/cells/mag.cpp:69-74), an NCCL all-reduce here --
 * and calls vgpu_dipole_finish, which computes the cell fields from the
 * sums.  While the field is pending the passes, vgpu_get_fields, the
 * statistics and Monte Carlo return VGPU_ERR_STATE. */
int vgpu_dipole_setup_shard(vgpu_handle h, const vgpu_dipole_desc* whole, int64_t n_global,
                            const int32_t* global_type, const int64_t* local);

/* Device buffer of the cell moments [3*num_cells FP64, J/T, x|y|z blocks]
 * (stream-ordered on vgpu_get_stream); *count = 3*num_cells. */
int vgpu_dipole_moment_buffer(vgpu_handle h, double** dev, int64_t* count);

/* *pending = 1 while a shard's cell moments await vgpu_dipole_finish. */
int vgpu_dipole_pending(vgpu_handle h, int32_t* pending);

/* Cell fields from the cell moments in the buffer (after their sum over
 * ranks); clears the pending state. */
int vgpu_dipole_finish(vgpu_handle h);

/* Far-field method chosen by vgpu_dipole_setup: VGPU_DIPOLE_FAR_DIRECT (tiled
 * all-pairs sum, FP32 terms) or VGPU_DIPOLE_FAR_FFT (FP64 FFT convolution on
 * the cell grid).  No reference counterpart: the reference stores dense
 * Nc x Nc tensors (src/dipole/memory.cpp:29-56). */
#define VGPU_DIPOLE_FAR_DIRECT 0
#define VGPU_DIPOLE_FAR_FFT 1
int vgpu_dipole_method(vgpu_handle h, int32_t* method);

/* Cell moments [3*num_cells, J/T, x|y|z], B field and mu0 Hd field
 * [3*num_cells, Tesla] of the last update (cells::mag_array_*,
 * dipole::cells_field_array_*, dipole::cells_mu0Hd_field_array_*); any
 * output may be NULL. */
int vgpu_dipole_get_cells(vgpu_handle h, double* mag, double* b_field, double* hd_field);

/* Host-computed per-atom dipole B field (and mu0 Hd field for energies; NULL
 * = zero): the reference's vcuda::transfer_dipole_fields_from_cpu_to_gpu
 * path, for hosts that keep the CPU dipole solver. */
int vgpu_set_dipole_field(vgpu_handle h, const double* bx, const double* by, const double* bz,
                          const double* hx, const double* hy, const double* hz);

/* ---- Metropolis Monte Carlo (checkerboard) ------------------------------ */

/* Colour the exchange graph for the parallel sweep: colour_in[num_atoms]
 * (checked: no two interacting atoms share a colour) or NULL for a host
 * greedy colouring.  The reference has no GPU Monte Carlo; this backs the
 * gpu::mc_step() entry the simulate loop gains (src/simulate/sim.cpp:608-614
 * calls montecarlo::mc_step, src/montecarlo/mc.cpp:29-127).  On a shard
 * (vgpu_set_owned, called first) the sweeps visit the owned atoms only; give
 * the whole system's colours of the local atoms (owned and halo) so that the
 * shards together make the whole system's sweep. */
int vgpu_mc_setup(vgpu_handle h, const int32_t* colour_in, int32_t* n_colours_out);

/* The colour of every atom chosen by vgpu_mc_setup. */
int vgpu_mc_get_colours(vgpu_handle h, int32_t* colour);

/* Replay mode: the next sweeps use these 4*num_atoms numbers (x|y|z move
 * Gaussians, then acceptance uniforms); NULL returns to Philox. */
int vgpu_mc_set_replay(vgpu_handle h, const double* rnd);

/* n_sweeps sweeps of angle moves (mc_angle, src/montecarlo/mc_moves.cpp:71-87,
 * sigma = 0.08 (kB T/muB)^0.2, or 0.02 below 1 K; mc.cpp:45-53) at the
 * temperature of vgpu_set_params; one launch per colour. */
int vgpu_mc_sweep(vgpu_handle h, uint64_t n_sweeps);

/* Sweep counter keying the Philox stream (counter = (noise_base + atom,
 * sweep), so shards draw the whole system's numbers). */
int vgpu_mc_set_sweep(vgpu_handle h, uint64_t sweep);

/* One colour of the current sweep, colours in order 0, 1, ...; the last one
 * completes the sweep.  For shards: between two colours the host refreshes
 * the halo spins (vgpu_halo_pack / vgpu_halo_unpack of VGPU_STATE_SPIN), the
 * exchange a colour-ordered sweep needs (the reference's parallel Monte
 * Carlo swaps halos around each of its eight octant phases,
 * src/montecarlo/mc-mpi.cpp:140-210).  No reference counterpart as an entry
 * point. */
int vgpu_mc_colour(vgpu_handle h, int32_t colour);

/* Attempted and rejected moves since vgpu_mc_setup
 * (sim::mc_statistics_moves / mc_statistics_reject). */
int vgpu_mc_counters(vgpu_handle h, double* moves, double* rejects);

/* ---- constrained Monte Carlo -------------------------------------------- */

/* Constrained Monte Carlo on the device.  Replaces montecarlo::cmc_step
 * (src/montecarlo/cmc.cpp:282-490), sim::integrate_serial case 3 (sim.cpp:
 * 623-629).  vgpu_cmc_setup sets the constraint direction (phi from z, theta
 * about z, in degrees: sim::constraint_phi, sim::constraint_theta; the frame
 * of polar_rot_matrix, cmc.cpp:53-135) and with init_spins != 0 turns every
 * spin along it (CMCinit); it colours the exchange graph if vgpu_mc_setup was
 * not called.  vgpu_cmc_sweep runs n_steps steps of about N pair moves each
 * (angle move of one spin, the second spin of the pair keeping the moment
 * perpendicular to the constraint, acceptance exp(-dE/kT) (Mz'/Mz)^2
 * |s2z/s2z'| with Mz' > 0): the pairs of a phase are atoms of one colour, so
 * their energy changes are independent and one warp accepts them in order
 * with the running total moment, the reference's rule.  The pairs differ from
 * the reference's random choice: the chains agree in distribution.
 * vgpu_cmc_pairs runs one phase on given pairs (2*num_pairs atoms, all of one
 * colour, each once) with given random numbers rnd[4*num_pairs] (the
 * Gaussians of the first spin's move, x|y|z blocks, then the acceptance
 * uniforms) from the total moment `moment` (mu_B; NULL: summed from the
 * spins).  vgpu_cmc_get: the running total moment (mu_B) and counters[4] =
 * pair moves, accepted, energy rejections, sphere rejections (cmc::mc_total,
 * mc_success, energy_reject, sphere_reject).  vgpu_cmc_frame: the rotation
 * P[9] (row-major, constraint direction to z) and the constraint vector. */
int vgpu_cmc_setup(vgpu_handle h, double phi_deg, double theta_deg, int32_t init_spins);
int vgpu_cmc_sweep(vgpu_handle h, uint64_t n_steps);
int vgpu_cmc_pairs(vgpu_handle h, const int32_t* pairs, int32_t num_pairs, const double* rnd, const double* moment);
int vgpu_cmc_get(vgpu_handle h, double* moment, double* counters);
int vgpu_cmc_frame(vgpu_handle h, double* P9, double* pv3);

/* Hybrid constrained Monte Carlo (montecarlo::cmc_mc_step, src/montecarlo/
 * cmc_mc.cpp:291-490; sim:integrator=hybrid-constrained-monte-carlo): each
 * material m with constrained[m] != 0 keeps its own moment along (phi_deg[m],
 * theta_deg[m]) (material[m]:constrained, constraint-angle-phi/theta), by
 * pair moves within that material against that material's running moment;
 * the other materials take single-spin Metropolis moves.  init_spins: the
 * constrained materials' spins along their directions (CMCMCinit).  Then
 * vgpu_cmc_sweep runs hybrid steps; vgpu_cmc_material_moments gives the
 * running moments [3*M] (mu_B) of the constrained materials. */
int vgpu_cmc_setup_materials(vgpu_handle h, const int32_t* constrained, const double* phi_deg, const double* theta_deg,
                             int32_t init_spins);
int vgpu_cmc_material_moments(vgpu_handle h, double* moments);

/* ---- statistics (masked reductions, FP64) -------------------------------- */

/* Register a statistics mask: mask[i] in [0, mask_size) is the bin of atom i
 * (the masks of magnetization_statistic_t::set_mask /
 * energy_statistic_t::set_mask, src/statistics/magnetization.cpp:54-116).
 * Returns its id.  Replaces the mask upload of vcuda::initialize
 * (src/cuda/initialize.cu:533-588). */
int vgpu_stats_add_mask(vgpu_handle h, const int32_t* mask, int32_t mask_size, int32_t* id_out);

/* Compute every registered mask on the device and add to the running means.
 * flags: bit 0 magnetisation (magnetization.cpp:134-180), bit 1 energy
 * (statistics/energy.cpp:141-258).  Replaces vcuda::stats::update
 * (src/cuda/statistics.cu:30-78), which computed magnetisation only. */
int vgpu_stats_update(vgpu_handle h, int32_t flags);

/* Magnetisation of mask `id`: m[4*bin + {0,1,2,3}] = (m_hat_x, m_hat_y,
 * m_hat_z, |m|/m_sat), empty bins zero; mean = running sum of those; counter =
 * number of updates summed.  Either output may be NULL.  Replaces
 * vcuda::stats::get (src/cuda/statistics.cu:252-284). */
int vgpu_stats_get_magnetization(vgpu_handle h, int32_t id, double* m, double* mean, int64_t* counter);

/* Energies of mask `id` in Tesla*muB: e[k*mask_size + bin], k = total,
 * exchange, anisotropy, applied, magnetostatic (exchange and magnetostatic
 * halved for the double sum); mean likewise. */
int vgpu_stats_get_energy(vgpu_handle h, int32_t id, double* e, double* mean, int64_t* counter);

/* Zero the running means and counters.  Replaces vcuda::stats::reset. */
int vgpu_stats_reset(vgpu_handle h);

/* Enqueue (no synchronisation) a copy of the latest finalised rows of mask
 * `id` into out[9*bin + k]: k = 0..3 magnetisation (m_hat, |m|/m_sat), 4..8
 * energies (total, exchange, anisotropy, applied, magnetostatic) -- the
 * values vgpu_stats_get_* return.  out is pinned host or device memory; the
 * copy completes in order on the handle's stream (vgpu_get_stream), so a
 * host can read step t's result while step t+1 runs.  Into pinned host
 * memory the device can address (cudaHostAlloc / cudaMallocHost under
 * unified addressing) the rows are written by a small kernel through that
 * mapping; otherwise by cudaMemcpyAsync.  No reference counterpart
 * (vcuda::stats::get blocks). */
int vgpu_stats_copy_rows(vgpu_handle h, int32_t id, double* out);

/* ---- spin snapshots (configuration output) ------------------------------ */

/* Output atom list of the spin snapshots: `count` atom ids (the reference's
 * config::internal::local_output_atom_list, built by config::internal::
 * initialize, src/config/initialize.cpp: atoms inside the output bounds), in
 * output order.  Replaces the host gather copy_data_to_buffer
 * (src/config/buffer.cpp:28-50) that config::internal::atoms
 * (src/config/atoms_spins.cpp) runs on every snapshot. */
int vgpu_snapshot_setup(vgpu_handle h, const int64_t* atoms, int64_t count);

/* Gather the listed atoms' spins on the device into the data block of the
 * binary spin file (src/config/write.cpp:107-140: x, y, z per atom, FP64) and
 * copy it to `out` (3 * count doubles, host memory; pinned memory makes the
 * copy asynchronous on the handle's stream -- call vgpu_synchronize before
 * reading it).  A file is a uint64 count followed by this block
 * (vampire_b200/config.py writes it with the reference's names and meta file). */
int vgpu_snapshot(vgpu_handle h, double* out);

/* Torque statistics.  Replaces stats::system_torque and stats::max_torque
 * (src/utility/statistics.cpp:221-325; output functions 14, 15 and 20 of
 * vio/outputfunctions.cpp).  vgpu_torque_update evaluates, from the current
 * spins and the total field H_i of every updated atom (spin fields plus
 * external fields: applied, thermal at the handle's current step, dipole),
 * T = sum_i mu_s,i S_i x H_i [J] for the system and per material, and
 * max_i |S_i x H_i| [T], and adds T to running sums; it runs on the handle's
 * stream without synchronising.  vgpu_torque_get (synchronises) returns
 * total[3], mean[3] (running sum / updates), material[3*M] and
 * material_mean[3*M] (x, y, z per material), max_torque and the update
 * count; any output may be NULL.  vgpu_torque_reset (also done by
 * vgpu_stats_reset, as the reference's mag_m_reset) zeroes the means.  On a
 * shard the sums cover the owned atoms; the host adds them over ranks. */
int vgpu_torque_update(vgpu_handle h);
int vgpu_torque_get(vgpu_handle h, double* total, double* mean, double* material, double* material_mean,
                    double* max_torque, int64_t* counter);
int vgpu_torque_reset(vgpu_handle h);

/* Raw per-bin sums of the last vgpu_stats_update of mask `id`: sums[8*bin +
 * {0..3}] = sum mu s_x, sum mu s_y, sum mu s_z, sum mu (mu_B), [4..7] = the
 * exchange, anisotropy, applied and magnetostatic energy sums (exchange and
 * magnetostatic before halving).  Shards add these over ranks and normalise
 * as magnetization.cpp:134-180.  No reference counterpart. */
int vgpu_stats_get_sums(vgpu_handle h, int32_t id, double* sums);

/* Derived statistics of mask `id` accumulated on the device at every
 * vgpu_stats_update since the last reset, evaluated as the reference's
 * output functions do at temperature T [K]: susceptibility[4*bin + {x,y,z,m}]
 * (statistics/susceptibility.cpp:70-88, from the magnetisation rows),
 * specific_heat[bin] (specific_heat.cpp:50-66, from the total energy; needs
 * energy updates) and std_dev[4*bin + {x,y,z,m}] (standard_deviation.cpp,
 * running Welford sums).  Any output may be NULL.  The reference computes
 * these on the host only and skips them in GPU mode (statistics.cpp:35-37). */
int vgpu_stats_get_derived(vgpu_handle h, int32_t id, double temperature, double* susceptibility,
                           double* specific_heat, double* std_dev);

/* ---- batched systems ------------------------------------------------------ */

/* No counterpart in the reference (one system per process there).  Per-system
 * parameters of a batch: temperature and a linear applied-field sweep
 * H(step) = H_start + (H_end - H_start) min(step, n_ramp)/n_ramp. */
typedef struct {
   double temperature;             /* [K]                                              */
   double H_start[3];              /* [T]                                              */
   double H_end[3];                /* [T]                                              */
   uint64_t n_ramp;                /* steps of the sweep (0: constant H_start)         */
} vgpu_batch_system;

/* One handle for n_sys independent systems of uneven sizes (same number of
 * materials and exchange type each).  The returned handle accepts the
 * single-system calls (vgpu_llg_heun steps all systems with two plain launches
 * per step; vgpu_get_spins returns all systems concatenated); system k's
 * Philox stream equals that of a single run seeded seed + k. */
int vgpu_batch_create(int device, int precision, int32_t n_sys, const vgpu_system_desc* descs,
                      const vgpu_batch_system* systems, const vgpu_sim_params* common, vgpu_handle* out);

/* Shape of the persistent launch: thread-block cluster size (1, 2, 4, 8) and
 * threads per block; systems are bin-packed onto the co-resident clusters.
 * cluster = 0 (block ignored): no persistent kernel -- vgpu_batch_run steps
 * the whole batch with the ordinary two passes per step (as vgpu_llg_heun),
 * with the same records; faster when one large system would dominate a
 * cluster's share.  Results are the same for every shape. */
int vgpu_batch_set_shape(vgpu_handle h, int32_t cluster, int32_t block);

/* Time every candidate shape (the step passes, cluster = 0, among them) for
 * trial_steps steps on this batch and keep the fastest (the state is
 * restored afterwards). */
int vgpu_batch_autotune(vgpu_handle h, int32_t trial_steps, int32_t* cluster_out, int32_t* block_out,
                        double* ms_per_step_out);

/* Advance n_steps with the persistent kernel (one launch per record_every
 * steps, or per 1000 when record_every is 0); record_every > 0 also stores
 * every system's magnetisation after each chunk; use_graph != 0 replays the
 * chunk as a CUDA graph. */
int vgpu_batch_run(vgpu_handle h, uint64_t n_steps, uint32_t record_every, int32_t use_graph);

/* Records of the last vgpu_batch_run: out[(r*n_sys + k)*4 + {0..3}] =
 * (m_hat_x, m_hat_y, m_hat_z, |m|/m_sat) of system k after record r. */
int vgpu_batch_history(vgpu_handle h, double* out, int64_t max_records, int64_t* n_records);

/* First atom and atom count of system k in the concatenated spin arrays. */
int vgpu_batch_system_range(vgpu_handle h, int32_t k, int32_t* first_atom, int32_t* num_atoms);

/* ---- adjoint (gradients of a trajectory loss) ----------------------------- */

/* No counterpart in the reference.  From the current spins (left unchanged),
 * run n_steps deterministic Heun steps and return
 *   loss = sum_{t=1..n_steps} w (m_z(t) - target[t-1])^2
 * (m_z: moment-weighted mean of s_z after step t) and
 *   grad[0] = dL/d(common scale of every exchange coupling),
 *   grad[1] = dL/dKu_SI (ku2 = Ku/mu_s), grad[2..4] = dL/dH_applied [1/T],
 * by the adjoint of the step with checkpoints every `every` steps
 * (0: ceil(sqrt(n_steps))).  Every exchange format (isotropic, vectorial,
 * diagonal + DMI, full tensor) and any number of materials, provided the
 * couplings are reciprocal in SI units (mu_s,j J_ji = (mu_s,i J_ij)^T, as a
 * symmetric exchange matrix and the three-site DMI give; checked on the
 * device, VGPU_ERR_ARG otherwise).  No thermal noise, no dipole field.  The
 * state, the recomputed steps and the adjoint vectors are in the handle's
 * precision (FP32 production, FP64 debug build); m_z, the loss and the
 * gradients are FP64 sums. */
int vgpu_adjoint_llg(vgpu_handle h, uint64_t n_steps, const double* target, double w, int32_t every,
                     double* loss_out, double* grad_out);

/* As vgpu_adjoint_llg, plus the gradients per pair of materials (at most 8
 * materials): pair_out[0] = dL/d(common scale of the DMI vectors) (0 without
 * an antisymmetric part), pair_out[1 + a*M + b] = dL/d(scale of the couplings
 * of the bonds from atoms of material a to atoms of material b) -- for the
 * diagonal + DMI format the diagonal, exchange-matrix part only.  Divided by
 * the exchange-matrix entry J_ab these are dL/dJ_ab, the gradients with
 * respect to the per-material exchange constants (material exchange-matrix,
 * exchange/interface.cpp:76-94).  pair_out holds 1 + M*M doubles. */
int vgpu_adjoint_llg_materials(vgpu_handle h, uint64_t n_steps, const double* target, double w, int32_t every,
                               double* loss_out, double* grad_out, double* pair_out);

/* m_z(t), t = 1..n_steps, of a deterministic run (the handle's precision,
 * FP64 sums) from the current spins (left unchanged): the targets of
 * vgpu_adjoint_llg. */
int vgpu_mz_trajectory(vgpu_handle h, uint64_t n_steps, double* mz_out);

/* ---- magnetisation without device allocation ----------------------------- */

/* No counterpart in the reference: an addition for callers that cannot call
 * cudaMalloc -- a plugin inside another framework whose caching allocator
 * owns the device memory (its own cudaMalloc would fragment that pool or fail
 * under the framework's memory cap), or a time-critical loop that must not
 * stall on the device synchronisation cudaMalloc/cudaFree can bring.  All
 * pointers are DEVICE pointers the caller owns: spins sx/sy/sz and moments
 * mu_muB [num_atoms] (FP32), mask [num_atoms] with bins in [0, mask_size)
 * (entries outside that range are skipped: counted in no bin), output m_out
 * [4*mask_size] (FP64: m_hat_x, m_hat_y, m_hat_z, |m|/m_sat per bin, empty
 * bins zero, as vgpu_stats_get_magnetization).  Runs on `stream` (a
 * cudaStream_t, NULL = default stream) and returns without synchronising; a
 * CUDA error already pending when it is called is returned, not launched over.
 * Scratch: a fixed array compiled into the library (VGPU_NOALLOC_MAX_BLOCKS x
 * VGPU_NOALLOC_MAX_BINS x 4 doubles = 512 KiB), held by every GPU that loads
 * the library until exit.  mask_size above VGPU_NOALLOC_MAX_BINS is refused
 * with VGPU_ERR_ARG.  The first call on a device looks up the array's device
 * address with that device current and keeps it for the process; make that
 * first call before any stream capture, and do not call it again on a device
 * after cudaDeviceReset.  Every call shares the one array (each call rewrites
 * the rows it reads, so nothing needs clearing): calls that overlap on the
 * GPU (other streams, other threads) race and must be serialised by the
 * caller. */
#define VGPU_NOALLOC_MAX_BLOCKS 256
#define VGPU_NOALLOC_MAX_BINS 64
int vgpu_magnetization_noalloc(const float* sx, const float* sy, const float* sz, const float* mu_muB,
                               const int32_t* mask, int32_t num_atoms, int32_t mask_size, double* m_out,
                               void* stream);

/* ---- streams, timing ----------------------------------------------------- */

/* The cudaStream_t (as void*) every call of this handle runs on. */
int vgpu_get_stream(vgpu_handle h, void** stream);

/* Wait for the handle's stream; reports VGPU_ERR_NAN if a pass flagged a
 * non-finite spin since the last check. */
int vgpu_synchronize(vgpu_handle h);

/* enable != 0: time every launch with CUDA events on the handle's stream
 * (resets the accumulators and the kernel-launch counter). */
int vgpu_profile(vgpu_handle h, int enable);

/* Accumulated device milliseconds and launch counts per kind
 * (0 predictor, 1 corrector, 2 statistics, 3 dipole, 4 Monte Carlo, 5 other)
 * and the number of kernels launched since vgpu_profile(). */
int vgpu_profile_read(vgpu_handle h, double* ms, int64_t* count, int32_t n_kinds, int64_t* kernel_launches);

#ifdef __cplusplus
}
#endif

#endif /* VGPU_H_ */
