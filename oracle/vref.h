/*
 * vref.h -- FP64 CPU restatement of the reference spin-update path.
 * TEST INFRASTRUCTURE ONLY (the oracle the CUDA path is checked against).
 */
#ifndef VREF_H_
#define VREF_H_
#include <stdint.h>

typedef struct {
   int n;                 /* atoms */
   int nmat;              /* materials */
   int exch_type;         /* 0 isotropic, 1 vectorial, 2 tensorial */
   int uniaxial, cubic;   /* anisotropy terms enabled */
   int thermal, applied;  /* hamiltonian_simulation_flags[3], [2] */
   int pad_;
   const int* start;      /* CSR: neighbour_list_start_index */
   const int* end;        /* CSR: neighbour_list_end_index (inclusive) */
   const int* nl;         /* neighbour_list_array */
   const int* nltype;     /* interaction id per bond, or NULL (= bond index) */
   const double* jlist;   /* per interaction: 1, 3 or 9 doubles [T] */
   const int* type;       /* material per atom */
   const double* A;       /* per material one_oneplusalpha_sq */
   const double* B;       /* per material alpha_oneplusalpha_sq */
   const double* sigma;   /* per material sqrt(T_rescaled) * H_th_sigma */
   const double* ku2;     /* per material reduced uniaxial constant [T] */
   const double* kux;
   const double* kuy;
   const double* kuz;
   const double* kc4;     /* per material reduced cubic constant [T] */
   double hx, hy, hz;     /* global applied field H_applied * H_vec [T] */
   const double* hloc;    /* per material local applied field (3 each) or NULL */
   const double* hdx;     /* per atom dipolar B field or NULL */
   const double* hdy;
   const double* hdz;
   const double* hmx;     /* per atom mu0 Hd field (magnetostatic energy) or NULL */
   const double* hmy;
   const double* hmz;
   double dt, half_dt;    /* reduced time step */
   double H_applied;      /* for the applied-field energy */
   double H_vec[3];
   const double* mus;     /* per material moment in mu_B (adjoint loss weights) */
   const double* mus_SI;  /* per material moment in J/T */
   /* higher-order anisotropy (src/anisotropy/internal.hpp) */
   int u4, u6, c6, crot, neel, pad2_;  /* enable_uniaxial_fourth/sixth_order, cubic_sixth_order,
                                         cubic_fourth_order_rotation, neel_anisotropy */
   const double* ku4;     /* per material reduced constants [T] */
   const double* ku6;
   const double* kc6;
   const double* kcb;     /* per material rotated cubic basis e1, e2, e3 (9 doubles) */
   const double* neelt;   /* per atom 3x3 Neel tensor (9 doubles), or NULL */
   /* biquadratic exchange (exchange/internal.hpp), NULL bq_start = off */
   const int* bq_start;
   const int* bq_end;     /* inclusive */
   const int* bq_nl;
   const int* bq_type;    /* interaction id per bond, or NULL (= bond index) */
   const double* bq_j;    /* isotropic J_bq [T] per interaction */
} vref_sys;

void vref_spin_fields(const vref_sys* s, const double* sx, const double* sy, const double* sz,
                      double* hx, double* hy, double* hz);
void vref_external_fields(const vref_sys* s, const double* xi, double* hx, double* hy, double* hz);
void vref_heun_predict(const vref_sys* s, const double* sx, const double* sy, const double* sz, const double* xi,
                       double* px, double* py, double* pz, double* keep);
void vref_heun_correct(const vref_sys* s, double* sx, double* sy, double* sz, const double* px, const double* py,
                       const double* pz, double* keep);
void vref_llg_heun_step(const vref_sys* s, double* sx, double* sy, double* sz, const double* xi,
                        double* work);
void vref_llg_midpoint_step(const vref_sys* s, double* sx, double* sy, double* sz, const double* xi,
                            const double* alpha, double* work);
void vref_llg_midpoint(const vref_sys* s, double* sx, double* sy, double* sz, const double* xi,
                       const double* alpha, int64_t n_steps);
void vref_llg_heun(const vref_sys* s, double* sx, double* sy, double* sz, const double* xi,
                   int64_t n_steps);
void vref_spin_energy(const vref_sys* s, const double* sx, const double* sy, const double* sz,
                      int atom, double Sx, double Sy, double Sz, double* e);
long vref_mc_colour_sweep(const vref_sys* s, double* sx, double* sy, double* sz, const int* order,
                          const int* colour_off, int ncolours, const double* rnd, const double* sigma,
                          const double* beta, const double* ratio);
double vref_adjoint(const vref_sys* s, const double* sx0, const double* sy0, const double* sz0, int64_t nsteps,
                    const double* target, double w, int64_t every, double* grad);
double vref_trajectory_loss(const vref_sys* s, const double* sx0, const double* sy0, const double* sz0,
                            int64_t nsteps, const double* target, double w);
void vref_mz_trajectory(const vref_sys* s, const double* sx0, const double* sy0, const double* sz0,
                        int64_t nsteps, double* mz_out);
void vref_magnetization(int n, const int* mask, int mask_size, const double* sx, const double* sy,
                        const double* sz, const double* mm, double* out);
void vref_energy(const vref_sys* s, const int* mask, int mask_size, const double* sx,
                 const double* sy, const double* sz, const double* mm, double* out);

#endif
