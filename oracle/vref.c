/*
 * vref.c -- FP64 CPU restatement of the reference VAMPIRE spin-update path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker that the CUDA path in vampire_b200 is
 * compared with.  Nothing in the product links or calls it.  It is pinned
 * against the reference itself: tests/golden/ holds fixtures produced by the
 * reference program (oracle/_ref/vampire-harness, reference objects built by
 * oracle/build_ref.py) and tests/test_oracle_pinned.py checks this file
 * against them.
 *
 * Each function follows the reference file:line cited beside it, with the
 * same operation order so that FP64 results agree to rounding.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "vref.h"

/* exchange::internal::exchange_fields (src/exchange/exchange_fields.cpp:29-168):
 * H_i += sum_j J_ij s_j over the CSR row [start, end] (end inclusive). */
static void exchange_fields(const vref_sys* s, const double* sx, const double* sy, const double* sz,
                            double* hx, double* hy, double* hz) {
   for (int atom = 0; atom < s->n; ++atom) {
      double fx = 0.0, fy = 0.0, fz = 0.0;
      const int start = s->start[atom];
      const int end = s->end[atom] + 1;
      for (int nn = start; nn < end; ++nn) {
         const int natom = s->nl[nn];
         const int iid = s->nltype ? s->nltype[nn] : nn;
         if (s->exch_type == 0) {
            const double J = s->jlist[iid];
            fx += J * sx[natom];
            fy += J * sy[natom];
            fz += J * sz[natom];
         } else if (s->exch_type == 1) {
            const double* J = s->jlist + 3 * (int64_t)iid;
            fx += J[0] * sx[natom];
            fy += J[1] * sy[natom];
            fz += J[2] * sz[natom];
         } else {
            const double* J = s->jlist + 9 * (int64_t)iid;
            const double S0 = sx[natom], S1 = sy[natom], S2 = sz[natom];
            fx += (J[0] * S0 + J[1] * S1 + J[2] * S2);
            fy += (J[3] * S0 + J[4] * S1 + J[5] * S2);
            fz += (J[6] * S0 + J[7] * S1 + J[8] * S2);
         }
      }
      hx[atom] += fx;
      hy[atom] += fy;
      hz[atom] += fz;
   }
}

/* calculate_spin_fields (src/simulate/fields.cpp:67-118): zero, exchange, then
 * anisotropy::fields -> uniaxial_second_order_fields
 * (src/anisotropy/uniaxial_second_order.cpp:51-98, H += 2 ku2 (s.e) e) and
 * cubic_fourth_order_fields (src/anisotropy/cubic_fourth_order.cpp:34-73,
 * H += 2 kc4 s^3). */
void vref_spin_fields(const vref_sys* s, const double* sx, const double* sy, const double* sz,
                      double* hx, double* hy, double* hz) {
   memset(hx, 0, sizeof(double) * s->n);
   memset(hy, 0, sizeof(double) * s->n);
   memset(hz, 0, sizeof(double) * s->n);
   exchange_fields(s, sx, sy, sz, hx, hy, hz);
   if (s->bq_start) {  /* exchange/biquadratic_fields.cpp:43-79 */
      for (int atom = 0; atom < s->n; atom++) {
         double bx = 0.0, by = 0.0, bz = 0.0;
         const double six = sx[atom], siy = sy[atom], siz = sz[atom];
         for (int nn = s->bq_start[atom]; nn < s->bq_end[atom] + 1; ++nn) {
            const int natom = s->bq_nl[nn];
            const double twoJbq = 2.0 * s->bq_j[s->bq_type ? s->bq_type[nn] : nn];
            const double sjx = sx[natom], sjy = sy[natom], sjz = sz[natom];
            const double si_dot_sj = six * sjx + siy * sjy + siz * sjz;
            bx += twoJbq * sjx * si_dot_sj;
            by += twoJbq * sjy * si_dot_sj;
            bz += twoJbq * sjz * si_dot_sj;
         }
         hx[atom] += bx;
         hy[atom] += by;
         hz[atom] += bz;
      }
   }
   if (s->uniaxial) {
      for (int atom = 0; atom < s->n; atom++) {
         const int mat = s->type[atom];
         const double ex = s->kux[mat], ey = s->kuy[mat], ez = s->kuz[mat];
         const double sdote = (sx[atom] * ex + sy[atom] * ey + sz[atom] * ez);
         const double k2 = 2.0 * s->ku2[mat] * sdote;
         hx[atom] += ex * k2;
         hy[atom] += ey * k2;
         hz[atom] += ez * k2;
      }
   }
   if (s->u4) {  /* uniaxial_fourth_order.cpp: H += (2/3)(1/8) ku4 (140 (s.e)^3 - 60 s.e) e */
      const double scale = 1.0 / 8.0 * 2.0 / 3.0;
      for (int atom = 0; atom < s->n; atom++) {
         const int mat = s->type[atom];
         const double ex = s->kux[mat], ey = s->kuy[mat], ez = s->kuz[mat];
         const double sdote = (sx[atom] * ex + sy[atom] * ey + sz[atom] * ez);
         const double sdote3 = sdote * sdote * sdote;
         const double k4 = scale * s->ku4[mat] * (140.0 * sdote3 - 60.0 * sdote);
         hx[atom] += ex * k4;
         hy[atom] += ey * k4;
         hz[atom] += ez * k4;
      }
   }
   if (s->u6) {  /* uniaxial_sixth_order.cpp: (2/3)(1/16) ku6 (1386 (s.e)^5 - 1260 (s.e)^3 + 210 s.e) e */
      const double scale = 1.0 / 16.0 * 2.0 / 3.0;
      for (int atom = 0; atom < s->n; atom++) {
         const int mat = s->type[atom];
         const double ex = s->kux[mat], ey = s->kuy[mat], ez = s->kuz[mat];
         const double sdote = (sx[atom] * ex + sy[atom] * ey + sz[atom] * ez);
         const double sdote3 = sdote * sdote * sdote;
         const double sdote5 = sdote3 * sdote * sdote;
         const double k6 = scale * s->ku6[mat] * (1386.0 * sdote5 - 1260.0 * sdote3 + 210.0 * sdote);
         hx[atom] += ex * k6;
         hy[atom] += ey * k6;
         hz[atom] += ez * k6;
      }
   }
   if (s->cubic) {
      for (int atom = 0; atom < s->n; atom++) {
         const int mat = s->type[atom];
         const double k4 = 0.5 * 4.0 * s->kc4[mat];
         const double x = sx[atom], y = sy[atom], z = sz[atom];
         hx[atom] += x * x * x * k4;
         hy[atom] += y * y * y * k4;
         hz[atom] += z * z * z * k4;
      }
   }
   if (s->crot) {  /* cubic_fourth_order_rotation.cpp: 2 kc4 sum_k (s.e_k)^3 e_k */
      for (int atom = 0; atom < s->n; atom++) {
         const int mat = s->type[atom];
         const double* e = s->kcb + 9 * mat;
         const double k4 = 0.5 * 4.0 * s->kc4[mat];
         const double x = sx[atom], y = sy[atom], z = sz[atom];
         const double d1 = x * e[0] + y * e[1] + z * e[2];
         const double d2 = x * e[3] + y * e[4] + z * e[5];
         const double d3 = x * e[6] + y * e[7] + z * e[8];
         const double d13 = d1 * d1 * d1, d23 = d2 * d2 * d2, d33 = d3 * d3 * d3;
         hx[atom] += k4 * (d13 * e[0] + d23 * e[3] + d33 * e[6]);
         hy[atom] += k4 * (d13 * e[1] + d23 * e[4] + d33 * e[7]);
         hz[atom] += k4 * (d13 * e[2] + d23 * e[5] + d33 * e[8]);
      }
   }
   if (s->c6) {  /* cubic_sixth_order.cpp: H_x += -2 kc6 s_x s_y^2 s_z^2 (cyclic) */
      for (int atom = 0; atom < s->n; atom++) {
         const int mat = s->type[atom];
         const double k6 = -2.0 * s->kc6[mat];
         const double x = sx[atom], y = sy[atom], z = sz[atom];
         const double x2 = x * x, y2 = y * y, z2 = z * z;
         hx[atom] += x * y2 * z2 * k6;
         hy[atom] += y * z2 * x2 * k6;
         hz[atom] += z * x2 * y2 * k6;
      }
   }
   if (s->neel && s->neelt) {  /* neel.cpp: H += 2 T s, per-atom tensor */
      for (int atom = 0; atom < s->n; atom++) {
         const double* t = s->neelt + 9 * (int64_t)atom;
         const double x = sx[atom], y = sy[atom], z = sz[atom];
         hx[atom] += 2.0 * (t[0] * x + t[1] * y + t[2] * z);
         hy[atom] += 2.0 * (t[3] * x + t[4] * y + t[5] * z);
         hz[atom] += 2.0 * (t[6] * x + t[7] * y + t[8] * z);
      }
   }
}

/* calculate_external_fields (src/simulate/fields.cpp:120-169): thermal
 * (246-289: xi * sqrt(T_resc) * H_th_sigma, xi in x|y|z blocks), applied
 * (171-244: global H plus optional per-material local field) and dipolar
 * (291-316: per-atom field).  sigma[mat] = sqrt(T_resc) * H_th_sigma. */
void vref_external_fields(const vref_sys* s, const double* xi, double* hx, double* hy, double* hz) {
   const int n = s->n;
   for (int atom = 0; atom < n; atom++) {
      if (xi && s->thermal) {
         const double sg = s->sigma[s->type[atom]];
         hx[atom] = xi[atom] * sg;
         hy[atom] = xi[n + atom] * sg;
         hz[atom] = xi[2 * n + atom] * sg;
      } else {
         hx[atom] = 0.0; hy[atom] = 0.0; hz[atom] = 0.0;
      }
   }
   if (s->applied) {
      for (int atom = 0; atom < n; atom++) {
         double ax = s->hx, ay = s->hy, az = s->hz;
         if (s->hloc) {
            const int m = s->type[atom];
            ax += s->hloc[3 * m + 0]; ay += s->hloc[3 * m + 1]; az += s->hloc[3 * m + 2];
         }
         hx[atom] += ax; hy[atom] += ay; hz[atom] += az;
      }
   }
   if (s->hdx) {
      for (int atom = 0; atom < n; atom++) {
         hx[atom] += s->hdx[atom]; hy[atom] += s->hdy[atom]; hz[atom] += s->hdz[atom];
      }
   }
}

/* Landau-Lifshitz-Gilbert right-hand side as written in LLGHeun.cpp:201-203. */
static inline void llg_rhs(double A, double B, const double S[3], const double H[3], double d[3]) {
   d[0] = A * (S[1] * H[2] - S[2] * H[1]) + B * (S[1] * (S[0] * H[1] - S[1] * H[0]) - S[2] * (S[2] * H[0] - S[0] * H[2]));
   d[1] = A * (S[2] * H[0] - S[0] * H[2]) + B * (S[2] * (S[1] * H[2] - S[2] * H[1]) - S[0] * (S[0] * H[1] - S[1] * H[0]));
   d[2] = A * (S[0] * H[1] - S[1] * H[0]) + B * (S[0] * (S[2] * H[0] - S[0] * H[2]) - S[1] * (S[1] * H[2] - S[2] * H[1]));
}

/* Predictor half of sim::LLG_Heun (src/simulate/LLGHeun.cpp:185-222): fields of
 * s0 (spin + external, LLGHeun.cpp:185-186), f0 = rhs(s0, H) kept in keep[6n..9n)
 * and the external field in keep[3n..6n) for the corrector, s' = n(s0 + f0 dt)
 * into px, py, pz.  keep: 12n doubles, passed unchanged to vref_heun_correct. */
void vref_heun_predict(const vref_sys* s, const double* sx, const double* sy, const double* sz, const double* xi,
                       double* px, double* py, double* pz, double* keep) {
   const int n = s->n;
   double* hsx = keep;          double* hsy = keep + n;      double* hsz = keep + 2 * n;
   double* hex = keep + 3 * n;  double* hey = keep + 4 * n;  double* hez = keep + 5 * n;
   double* ex = keep + 6 * n;   double* ey = keep + 7 * n;   double* ez = keep + 8 * n;
   vref_spin_fields(s, sx, sy, sz, hsx, hsy, hsz);
   vref_external_fields(s, xi, hex, hey, hez);
   for (int atom = 0; atom < n; atom++) {
      const int m = s->type[atom];
      const double S[3] = {sx[atom], sy[atom], sz[atom]};
      const double H[3] = {hsx[atom] + hex[atom], hsy[atom] + hey[atom], hsz[atom] + hez[atom]};
      double d[3];
      llg_rhs(s->A[m], s->B[m], S, H, d);
      ex[atom] = d[0]; ey[atom] = d[1]; ez[atom] = d[2];
      double Sn[3] = {S[0] + d[0] * s->dt, S[1] + d[1] * s->dt, S[2] + d[2] * s->dt};
      const double mod = 1.0 / sqrt(Sn[0] * Sn[0] + Sn[1] * Sn[1] + Sn[2] * Sn[2]);
      px[atom] = Sn[0] * mod; py[atom] = Sn[1] * mod; pz[atom] = Sn[2] * mod;
   }
}

/* Corrector half (LLGHeun.cpp:224-279): spin fields of s' plus the predictor's
 * external field (the same thermal field serves both halves, LLGHeun.cpp:185),
 * f1 = rhs(s', H'), s1 = n(s0 + dt/2 (f0 + f1)) written over sx, sy, sz (s0). */
void vref_heun_correct(const vref_sys* s, double* sx, double* sy, double* sz, const double* px, const double* py,
                       const double* pz, double* keep) {
   const int n = s->n;
   double* hsx = keep;          double* hsy = keep + n;      double* hsz = keep + 2 * n;
   double* hex = keep + 3 * n;  double* hey = keep + 4 * n;  double* hez = keep + 5 * n;
   double* ex = keep + 6 * n;   double* ey = keep + 7 * n;   double* ez = keep + 8 * n;
   double* hux = keep + 9 * n;  double* huy = keep + 10 * n; double* huz = keep + 11 * n;
   vref_spin_fields(s, px, py, pz, hsx, hsy, hsz);
   for (int atom = 0; atom < n; atom++) {
      const int m = s->type[atom];
      const double S[3] = {px[atom], py[atom], pz[atom]};
      const double H[3] = {hsx[atom] + hex[atom], hsy[atom] + hey[atom], hsz[atom] + hez[atom]};
      double d[3];
      llg_rhs(s->A[m], s->B[m], S, H, d);
      hux[atom] = d[0]; huy[atom] = d[1]; huz[atom] = d[2];
   }
   for (int atom = 0; atom < n; atom++) {
      double Sn[3] = {sx[atom] + s->half_dt * (ex[atom] + hux[atom]),
                      sy[atom] + s->half_dt * (ey[atom] + huy[atom]),
                      sz[atom] + s->half_dt * (ez[atom] + huz[atom])};
      const double mod = 1.0 / sqrt(Sn[0] * Sn[0] + Sn[1] * Sn[1] + Sn[2] * Sn[2]);
      sx[atom] = Sn[0] * mod; sy[atom] = Sn[1] * mod; sz[atom] = Sn[2] * mod;
   }
}

/* sim::LLG_Heun (src/simulate/LLGHeun.cpp:160-282): one stochastic Heun step.
 * xi: 3n Gaussians for this step (NULL = no thermal term).  work: 15n doubles. */
void vref_llg_heun_step(const vref_sys* s, double* sx, double* sy, double* sz, const double* xi,
                        double* work) {
   const int n = s->n;
   double* px = work + 12 * n;  double* py = work + 13 * n;  double* pz = work + 14 * n;
   vref_heun_predict(s, sx, sy, sz, xi, px, py, pz, work);
   vref_heun_correct(s, sx, sy, sz, px, py, pz, work);
}

/* Cayley-transform rotation of sim::LLG_Midpoint (src/simulate/LLGMidpoint.cpp:
 * 70-105 and 117-150): with F = H + alpha M x H and beta = -dt A / 2,
 * out = (S (1 - b2 F.F) + 2 (beta F x S + F b2 F.S)) / (1 + b2 F.F), b2 = beta^2. */
static inline void midpoint_rotate(double alpha, double beta, const double M[3], const double S[3],
                                   const double H[3], double out[3]) {
   const double beta2 = beta * beta;
   const double F[3] = {H[0] + alpha * (M[1] * H[2] - M[2] * H[1]),
                        H[1] + alpha * (M[2] * H[0] - M[0] * H[2]),
                        H[2] + alpha * (M[0] * H[1] - M[1] * H[0])};
   const double FdotF = F[0] * F[0] + F[1] * F[1] + F[2] * F[2];
   const double beta2FdotS = beta2 * (F[0] * S[0] + F[1] * S[1] + F[2] * S[2]);
   const double c1 = 1.0 / (1.0 + beta2 * FdotF);
   const double c2 = 1.0 - beta2 * FdotF;
   out[0] = c1 * (S[0] * c2 + 2.0 * (beta * (F[1] * S[2] - F[2] * S[1]) + F[0] * beta2FdotS));
   out[1] = c1 * (S[1] * c2 + 2.0 * (beta * (F[2] * S[0] - F[0] * S[2]) + F[1] * beta2FdotS));
   out[2] = c1 * (S[2] * c2 + 2.0 * (beta * (F[0] * S[1] - F[1] * S[0]) + F[2] * beta2FdotS));
}

/* sim::LLG_Midpoint (src/simulate/LLGMidpoint.cpp:48-150): midpoint
 * M = (S + R(S; F(S, H(S)))) / 2 (not renormalised), then
 * S1 = R(S; F(M, H_spin(M) + H_ext)) with the external field of the first half.
 * work: 12n doubles. */
void vref_llg_midpoint_step(const vref_sys* s, double* sx, double* sy, double* sz, const double* xi,
                            const double* alpha, double* work) {
   const int n = s->n;
   double* hsx = work;          double* hsy = work + n;      double* hsz = work + 2 * n;
   double* hex = work + 3 * n;  double* hey = work + 4 * n;  double* hez = work + 5 * n;
   double* ix = work + 6 * n;   double* iy = work + 7 * n;   double* iz = work + 8 * n;
   double* mx = work + 9 * n;   double* my = work + 10 * n;  double* mz = work + 11 * n;
   memcpy(ix, sx, sizeof(double) * n);
   memcpy(iy, sy, sizeof(double) * n);
   memcpy(iz, sz, sizeof(double) * n);
   vref_spin_fields(s, sx, sy, sz, hsx, hsy, hsz);
   vref_external_fields(s, xi, hex, hey, hez);
   for (int atom = 0; atom < n; atom++) {
      const int m = s->type[atom];
      const double beta = -1.0 * s->dt * s->A[m] * 0.5;
      const double S[3] = {sx[atom], sy[atom], sz[atom]};
      const double H[3] = {hsx[atom] + hex[atom], hsy[atom] + hey[atom], hsz[atom] + hez[atom]};
      double R[3];
      midpoint_rotate(alpha[m], beta, S, S, H, R);
      mx[atom] = (S[0] + R[0]) * 0.5;
      my[atom] = (S[1] + R[1]) * 0.5;
      mz[atom] = (S[2] + R[2]) * 0.5;
   }
   vref_spin_fields(s, mx, my, mz, hsx, hsy, hsz);
   for (int atom = 0; atom < n; atom++) {
      const int m = s->type[atom];
      const double beta = -1.0 * s->dt * s->A[m] * 0.5;
      const double M[3] = {mx[atom], my[atom], mz[atom]};
      const double S[3] = {ix[atom], iy[atom], iz[atom]};
      const double H[3] = {hsx[atom] + hex[atom], hsy[atom] + hey[atom], hsz[atom] + hez[atom]};
      double R[3];
      midpoint_rotate(alpha[m], beta, M, S, H, R);
      sx[atom] = R[0]; sy[atom] = R[1]; sz[atom] = R[2];
   }
}

void vref_llg_midpoint(const vref_sys* s, double* sx, double* sy, double* sz, const double* xi,
                       const double* alpha, int64_t n_steps) {
   double* work = (double*)malloc(sizeof(double) * 12 * (size_t)s->n);
   for (int64_t t = 0; t < n_steps; t++)
      vref_llg_midpoint_step(s, sx, sy, sz, xi ? xi + t * 3 * (int64_t)s->n : NULL, alpha, work);
   free(work);
}

/* n_steps deterministic (T=0 or given-noise) steps; xi may be NULL or hold
 * n_steps * 3n values. */
void vref_llg_heun(const vref_sys* s, double* sx, double* sy, double* sz, const double* xi,
                   int64_t n_steps) {
   double* work = (double*)malloc(sizeof(double) * 15 * (size_t)s->n);
   for (int64_t t = 0; t < n_steps; t++)
      vref_llg_heun_step(s, sx, sy, sz, xi ? xi + t * 3 * (int64_t)s->n : NULL, work);
   free(work);
}

/* Energies of one spin in Tesla, as sim::calculate_spin_energy
 * (src/simulate/energy.cpp:147-174): exchange (exchange/energy.cpp:27-140),
 * anisotropy (uniaxial_second_order.cpp:104-121: -ku2 (s.e)^2;
 * cubic_fourth_order.cpp:80-95: -kc4/2 sum s^4), applied (-H.s) and
 * magnetostatic (-Hd.s).  Out: e[0]=exchange, [1]=anisotropy, [2]=applied,
 * [3]=magnetostatic. */
void vref_spin_energy(const vref_sys* s, const double* sx, const double* sy, const double* sz,
                      int atom, double Sx, double Sy, double Sz, double* e) {
   double ex = 0.0;
   for (int nn = s->start[atom]; nn <= s->end[atom]; ++nn) {
      const int natom = s->nl[nn];
      const int iid = s->nltype ? s->nltype[nn] : nn;
      if (s->exch_type == 0) {
         const double J = s->jlist[iid];
         ex -= J * (sx[natom] * Sx + sy[natom] * Sy + sz[natom] * Sz);
      } else if (s->exch_type == 1) {
         const double* J = s->jlist + 3 * (int64_t)iid;
         ex -= (J[0] * sx[natom] * Sx + J[1] * sy[natom] * Sy + J[2] * sz[natom] * Sz);
      } else {
         const double* J = s->jlist + 9 * (int64_t)iid;
         const double S0 = sx[natom], S1 = sy[natom], S2 = sz[natom];
         ex -= (J[0] * S0 * Sx + J[1] * S1 * Sx + J[2] * S2 * Sx + J[3] * S0 * Sy + J[4] * S1 * Sy +
                J[5] * S2 * Sy + J[6] * S0 * Sz + J[7] * S1 * Sz + J[8] * S2 * Sz);
      }
   }
   if (s->bq_start) {  /* exchange/biquadratic_energy.cpp:24-37 */
      double eb = 0.0;
      for (int nn = s->bq_start[atom]; nn <= s->bq_end[atom]; ++nn) {
         const int natom = s->bq_nl[nn];
         const double Jbq = s->bq_j[s->bq_type ? s->bq_type[nn] : nn];
         const double d = Sx * sx[natom] + Sy * sy[natom] + Sz * sz[natom];
         eb -= Jbq * d * d;
      }
      ex += eb;
   }
   const int m = s->type[atom];
   double an = 0.0;
   if (s->uniaxial) {
      const double sdote = Sx * s->kux[m] + Sy * s->kuy[m] + Sz * s->kuz[m];
      an += -s->ku2[m] * (sdote * sdote);
   }
   if (s->u4) {  /* uniaxial_fourth_order.cpp energy (the reference's literal 1/12) */
      const double sdote = Sx * s->kux[m] + Sy * s->kuy[m] + Sz * s->kuz[m];
      const double sdote2 = sdote * sdote;
      an += -0.08333333333 * s->ku4[m] * (35.0 * sdote2 * sdote2 - 30.0 * sdote2);
   }
   if (s->u6) {  /* uniaxial_sixth_order.cpp energy (literal 1/24) */
      const double sdote = Sx * s->kux[m] + Sy * s->kuy[m] + Sz * s->kuz[m];
      const double sdote2 = sdote * sdote;
      an += -0.04166666666 * s->ku6[m] * (231.0 * sdote2 * sdote2 * sdote2 - 315.0 * sdote2 * sdote2 + 105.0 * sdote2);
   }
   if (s->cubic) {
      const double sx4 = Sx * Sx * Sx * Sx, sy4 = Sy * Sy * Sy * Sy, sz4 = Sz * Sz * Sz * Sz;
      an += -0.5 * s->kc4[m] * (sx4 + sy4 + sz4);
   }
   if (s->crot) {
      const double* e = s->kcb + 9 * m;
      const double d1 = Sx * e[0] + Sy * e[1] + Sz * e[2];
      const double d2 = Sx * e[3] + Sy * e[4] + Sz * e[5];
      const double d3 = Sx * e[6] + Sy * e[7] + Sz * e[8];
      const double x4 = d1 * d1 * d1 * d1, y4 = d2 * d2 * d2 * d2, z4 = d3 * d3 * d3 * d3;
      an += -0.5 * s->kc4[m] * (x4 + y4 + z4);
   }
   if (s->c6) an += s->kc6[m] * Sx * Sx * Sy * Sy * Sz * Sz;
   if (s->neel && s->neelt) {
      const double* t = s->neelt + 9 * (int64_t)atom;
      const double en = (Sx * t[0] * Sx + Sx * t[1] * Sy + Sx * t[2] * Sz + Sy * t[3] * Sx + Sy * t[4] * Sy +
                         Sy * t[5] * Sz + Sz * t[6] * Sx + Sz * t[7] * Sy + Sz * t[8] * Sz);
      an += -1.0 * en;
   }
   e[0] = ex;
   e[1] = an;
   e[2] = -s->H_applied * (s->H_vec[0] * Sx + s->H_vec[1] * Sy + s->H_vec[2] * Sz);
   e[3] = s->hmx ? -(s->hmx[atom] * Sx + s->hmy[atom] * Sy + s->hmz[atom] * Sz) : 0.0;
}

/* One colour-ordered Metropolis sweep with given random numbers: the
 * reference's per-trial rule (montecarlo::mc_step, src/montecarlo/mc.cpp:59-110,
 * mc_angle, src/montecarlo/mc_moves.cpp:71-87) applied to the sites of
 * colour 0, then colour 1, ... (order[colour_off[c] .. colour_off[c+1]]).
 * rnd: 4n values, x|y|z Gaussians then the acceptance uniform, per site.
 * sigma/beta/ratio per material: move width, muB/(kB T), mu_s/muB.
 * Returns the number of rejected trials. */
long vref_mc_colour_sweep(const vref_sys* s, double* sx, double* sy, double* sz, const int* order,
                          const int* colour_off, int ncolours, const double* rnd, const double* sigma,
                          const double* beta, const double* ratio) {
   const int n = s->n;
   long rejects = 0;
   for (int c = 0; c < ncolours; ++c) {
      for (int k = colour_off[c]; k < colour_off[c + 1]; ++k) {
         const int atom = order[k];
         const int m = s->type[atom];
         const double S[3] = {sx[atom], sy[atom], sz[atom]};
         double T[3] = {S[0] + rnd[atom] * sigma[m], S[1] + rnd[n + atom] * sigma[m], S[2] + rnd[2 * n + atom] * sigma[m]};
         const double r = 1.0 / sqrt(T[0] * T[0] + T[1] * T[1] + T[2] * T[2]);
         T[0] *= r; T[1] *= r; T[2] *= r;
         double eo[4], en[4];
         vref_spin_energy(s, sx, sy, sz, atom, S[0], S[1], S[2], eo);
         vref_spin_energy(s, sx, sy, sz, atom, T[0], T[1], T[2], en);
         const double Eold = eo[0] + eo[1] + eo[2] + eo[3];
         const double Enew = en[0] + en[1] + en[2] + en[3];
         const double DE = (Enew - Eold) * ratio[m];
         int accept = DE < 0;
         if (!accept) accept = exp(-DE * beta[m]) >= rnd[3 * n + atom];
         if (accept) {
            sx[atom] = T[0]; sy[atom] = T[1]; sz[atom] = T[2];
         } else {
            rejects++;
         }
      }
   }
   return rejects;
}

/* Constrained Monte Carlo pair moves, the rule of montecarlo::cmc_step
 * (src/montecarlo/cmc.cpp:282-490) applied to a given ordered list of pairs
 * (pairs[2k], pairs[2k+1]) with given random numbers rnd[4K] (Gaussians of
 * the angle move of the first spin in x|y|z blocks of K, then the acceptance
 * uniforms).  In the frame P (rows: P s rotates the constraint direction to
 * z; pv the constraint direction) the second spin takes the perpendicular
 * moment change of the first (scaled by mu1/mu2) so that the moment
 * perpendicular to pv is kept, its parallel component from |s| = 1 with its
 * sign kept; rejected outright when that leaves the unit sphere.  Accepted if
 * exp(-dE) (Mz'/Mz)^2 |s2z/s2z'| >= U and Mz' > 0; M (3, mu_B) is the running
 * total moment.  counts: [accepted, energy rejections, sphere rejections]. */
void vref_cmc_pairs(const vref_sys* s, double* sx, double* sy, double* sz, const int* pairs, int K,
                    const double* rnd, const double* P, const double* pv, double* M, const double* sigma,
                    const double* beta, const double* ratio, long* counts) {
   for (int k = 0; k < K; ++k) {
      const int a1 = pairs[2 * k], a2 = pairs[2 * k + 1];
      const int m1 = s->type[a1], m2 = s->type[a2];
      const double mu1 = ratio[m1], mu2 = ratio[m2];
      const double s1i[3] = {sx[a1], sy[a1], sz[a1]};
      double s1f[3] = {s1i[0] + rnd[k] * sigma[m1], s1i[1] + rnd[K + k] * sigma[m1], s1i[2] + rnd[2 * K + k] * sigma[m1]};
      const double r = 1.0 / sqrt(s1f[0] * s1f[0] + s1f[1] * s1f[1] + s1f[2] * s1f[2]);
      s1f[0] *= r; s1f[1] *= r; s1f[2] *= r;
      double s1im[3], s1fm[3], s2im[3], s2fm[3];
      for (int q = 0; q < 3; ++q) {
         s1im[q] = P[3 * q] * s1i[0] + P[3 * q + 1] * s1i[1] + P[3 * q + 2] * s1i[2];
         s1fm[q] = P[3 * q] * s1f[0] + P[3 * q + 1] * s1f[1] + P[3 * q + 2] * s1f[2];
      }
      double eo[4], en[4];
      vref_spin_energy(s, sx, sy, sz, a1, s1i[0], s1i[1], s1i[2], eo);
      sx[a1] = s1f[0]; sy[a1] = s1f[1]; sz[a1] = s1f[2];
      vref_spin_energy(s, sx, sy, sz, a1, s1f[0], s1f[1], s1f[2], en);
      const double de1 = ((en[0] + en[1] + en[2] + en[3]) - (eo[0] + eo[1] + eo[2] + eo[3])) * ratio[m1];
      const double s2i[3] = {sx[a2], sy[a2], sz[a2]};
      for (int q = 0; q < 3; ++q) s2im[q] = P[3 * q] * s2i[0] + P[3 * q + 1] * s2i[1] + P[3 * q + 2] * s2i[2];
      const double mr = mu1 / mu2;
      s2fm[0] = mr * (s1im[0] - s1fm[0]) + s2im[0];
      s2fm[1] = mr * (s1im[1] - s1fm[1]) + s2im[1];
      if ((s2fm[0] * s2fm[0] + s2fm[1] * s2fm[1]) < 1.0 && a1 != a2) {
         s2fm[2] = (s2im[2] >= 0.0 ? 1.0 : -1.0) * sqrt(1.0 - s2fm[0] * s2fm[0] - s2fm[1] * s2fm[1]);
         double s2f[3];
         for (int q = 0; q < 3; ++q) s2f[q] = P[q] * s2fm[0] + P[3 + q] * s2fm[1] + P[6 + q] * s2fm[2];
         vref_spin_energy(s, sx, sy, sz, a2, s2i[0], s2i[1], s2i[2], eo);
         sx[a2] = s2f[0]; sy[a2] = s2f[1]; sz[a2] = s2f[2];
         vref_spin_energy(s, sx, sy, sz, a2, s2f[0], s2f[1], s2f[2], en);
         const double de2 = ((en[0] + en[1] + en[2] + en[3]) - (eo[0] + eo[1] + eo[2] + eo[3])) * ratio[m2];
         const double de21 = de1 * beta[m1] + de2 * beta[m2];
         const double mzo = M[0] * pv[0] + M[1] * pv[1] + M[2] * pv[2];
         double mn[3];
         for (int q = 0; q < 3; ++q) mn[q] = M[q] + mu1 * s1f[q] + mu2 * s2f[q] - mu1 * s1i[q] - mu2 * s2i[q];
         const double mzn = mn[0] * pv[0] + mn[1] * pv[1] + mn[2] * pv[2];
         const double prob = exp(-de21) * ((mzn / mzo) * (mzn / mzo)) * fabs(s2im[2] / s2fm[2]);
         if (prob >= rnd[3 * K + k] && mzn > 0.0) {
            M[0] = mn[0]; M[1] = mn[1]; M[2] = mn[2];
            counts[0]++;
         } else {
            sx[a1] = s1i[0]; sy[a1] = s1i[1]; sz[a1] = s1i[2];
            sx[a2] = s2i[0]; sy[a2] = s2i[1]; sz[a2] = s2i[2];
            counts[1]++;
         }
      } else {
         sx[a1] = s1i[0]; sy[a1] = s1i[1]; sz[a1] = s1i[2];
         counts[2]++;
      }
   }
}

/* ------------------------------------------------------------------------
 * FP64 CPU adjoint of the deterministic Heun step (no reference counterpart:
 * the reference has no derivatives).  Loss L = sum_{t=1..N} w (m_z(t) - T_t)^2
 * with m_z the moment-weighted mean of s_z and w the physical time step.
 * Gradients: dL/d(scale of every exchange coupling), dL/dKu_SI (ku2 = Ku/mu_s),
 * dL/dH_applied (3 components, Tesla).  Any exchange type and material
 * set whose couplings are reciprocal in SI units (mu_s,j J_ji = (mu_s,i
 * J_ij)^T, as the reference's symmetric exchange matrix and three-site DMI
 * give): the transposed gather sum_j J_ji^T Hbar_j is then mu_s,i times the
 * gather of Hbar / mu_s.  Checkpoints every `every` steps, states recomputed
 * per segment.
 * ---------------------------------------------------------------------- */
static void exch_only(const vref_sys* s, const double* x, const double* y, const double* z, double* hx,
                      double* hy, double* hz) {
   memset(hx, 0, sizeof(double) * s->n);
   memset(hy, 0, sizeof(double) * s->n);
   memset(hz, 0, sizeof(double) * s->n);
   exchange_fields(s, x, y, z, hx, hy, hz);
}

/* sum_j J_ji^T hb_j = mu_s,i sum_j J_ij (hb_j / mu_s,j) for reciprocal couplings */
static void exch_transposed(const vref_sys* s, const double* hb, double* out, double* scratch) {
   const int n = s->n;
   for (int i = 0; i < n; ++i) {
      const double r = 1.0 / s->mus[s->type[i]];
      for (int k = 0; k < 3; ++k) scratch[k * n + i] = hb[k * n + i] * r;
   }
   exch_only(s, scratch, scratch + n, scratch + 2 * n, out, out + n, out + 2 * n);
   for (int i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) out[k * n + i] *= s->mus[s->type[i]];
}

static void aniso_field(const vref_sys* s, int i, const double S[3], double H[3]) {
   const int m = s->type[i];
   H[0] = H[1] = H[2] = 0.0;
   if (s->uniaxial) {
      const double e[3] = {s->kux[m], s->kuy[m], s->kuz[m]};
      const double k2 = 2.0 * s->ku2[m] * (S[0] * e[0] + S[1] * e[1] + S[2] * e[2]);
      H[0] += e[0] * k2; H[1] += e[1] * k2; H[2] += e[2] * k2;
   }
   if (s->cubic) {
      const double k4 = 2.0 * s->kc4[m];
      H[0] += S[0] * S[0] * S[0] * k4; H[1] += S[1] * S[1] * S[1] * k4; H[2] += S[2] * S[2] * S[2] * k4;
   }
}

/* vector-Jacobian products of f(s,H) = A s x H + B s x (s x H) */
static void f_vjp(double A, double B, const double s[3], const double H[3], const double a[3], double sb[3],
                  double Hb[3]) {
   const double sH = s[0] * H[0] + s[1] * H[1] + s[2] * H[2];
   const double as = a[0] * s[0] + a[1] * s[1] + a[2] * s[2];
   const double aH = a[0] * H[0] + a[1] * H[1] + a[2] * H[2];
   const double ss = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
   /* A s x H: d/ds = H x a, d/dH = a x s */
   sb[0] = A * (H[1] * a[2] - H[2] * a[1]);
   sb[1] = A * (H[2] * a[0] - H[0] * a[2]);
   sb[2] = A * (H[0] * a[1] - H[1] * a[0]);
   Hb[0] = A * (a[1] * s[2] - a[2] * s[1]);
   Hb[1] = A * (a[2] * s[0] - a[0] * s[2]);
   Hb[2] = A * (a[0] * s[1] - a[1] * s[0]);
   /* B (s (s.H) - H (s.s)) */
   for (int k = 0; k < 3; ++k) {
      sb[k] += B * (a[k] * sH + as * H[k] - 2.0 * aH * s[k]);
      Hb[k] += B * (as * s[k] - a[k] * ss);
   }
}

static void f_eval(double A, double B, const double S[3], const double H[3], double d[3]) {
   llg_rhs(A, B, S, H, d);
}

double vref_adjoint(const vref_sys* s, const double* sx0, const double* sy0, const double* sz0, int64_t nsteps,
                    const double* target, double w, int64_t every, double* grad) {
   const int n = s->n;
   const double dt = s->dt;
   const double Happ[3] = {s->hx, s->hy, s->hz};
   double musum = 0.0;
   for (int i = 0; i < n; ++i) musum += s->mus[s->type[i]];
   if (every <= 0) every = (int64_t)ceil(sqrt((double)nsteps));
   const int64_t ncp = (nsteps + every - 1) / every;
   double* cp = (double*)malloc(sizeof(double) * 3 * n * (ncp + 1));
   double* seg = (double*)malloc(sizeof(double) * 3 * n * (every + 1));
   double* mz = (double*)malloc(sizeof(double) * (nsteps + 1));
   double* work = (double*)malloc(sizeof(double) * 15 * n);
   double* cur = (double*)malloc(sizeof(double) * 3 * n);
   memcpy(cur, sx0, sizeof(double) * n);
   memcpy(cur + n, sy0, sizeof(double) * n);
   memcpy(cur + 2 * n, sz0, sizeof(double) * n);
   /* forward with checkpoints and m_z(t) */
   double loss = 0.0;
   for (int64_t t = 0; t < nsteps; ++t) {
      if (t % every == 0) memcpy(cp + 3 * n * (t / every), cur, sizeof(double) * 3 * n);
      vref_llg_heun_step(s, cur, cur + n, cur + 2 * n, NULL, work);
      double m = 0.0;
      for (int i = 0; i < n; ++i) m += s->mus[s->type[i]] * cur[2 * n + i];
      mz[t + 1] = m / musum;
      const double r = mz[t + 1] - target[t];
      loss += w * r * r;
   }
   /* backward */
   double* lam = (double*)calloc(3 * n, sizeof(double));
   double* ex0 = (double*)malloc(sizeof(double) * 3 * n);
   double* ex1 = (double*)malloc(sizeof(double) * 3 * n);
   double* sp = (double*)malloc(sizeof(double) * 3 * n);
   double* Hb1 = (double*)malloc(sizeof(double) * 3 * n);
   double* Hb0 = (double*)malloc(sizeof(double) * 3 * n);
   double* tmp = (double*)malloc(sizeof(double) * 3 * n);
   double* spb = (double*)malloc(sizeof(double) * 3 * n);
   double* sb = (double*)malloc(sizeof(double) * 3 * n);
   double* ub = (double*)malloc(sizeof(double) * 3 * n);
   double* f0 = (double*)malloc(sizeof(double) * 3 * n);
   double* nv = (double*)malloc(sizeof(double) * n);
   double* f1s = (double*)malloc(sizeof(double) * 3 * n);
   double gJ = 0.0, gK = 0.0, gH[3] = {0, 0, 0};
   /* lambda_N = dL_N/ds_N */
   for (int i = 0; i < n; ++i) lam[2 * n + i] = 2.0 * w * (mz[nsteps] - target[nsteps - 1]) * s->mus[s->type[i]] / musum;
   for (int64_t c = ncp - 1; c >= 0; --c) {
      const int64_t t0 = c * every, t1 = (t0 + every < nsteps) ? t0 + every : nsteps;
      memcpy(seg, cp + 3 * n * c, sizeof(double) * 3 * n);
      for (int64_t t = t0; t < t1 - 1; ++t) {
         double* a = seg + 3 * n * (t - t0);
         double* b = seg + 3 * n * (t - t0 + 1);
         memcpy(b, a, sizeof(double) * 3 * n);
         vref_llg_heun_step(s, b, b + n, b + 2 * n, NULL, work);
      }
      for (int64_t t = t1 - 1; t >= t0; --t) {
         const double* S = seg + 3 * n * (t - t0);
         /* recompute the step from S */
         exch_only(s, S, S + n, S + 2 * n, ex0, ex0 + n, ex0 + 2 * n);
         for (int i = 0; i < n; ++i) {
            const int m = s->type[i];
            const double Si[3] = {S[i], S[n + i], S[2 * n + i]};
            double Ha[3], H[3], d[3];
            aniso_field(s, i, Si, Ha);
            for (int k = 0; k < 3; ++k) H[k] = ex0[k * n + i] + Ha[k] + Happ[k];
            f_eval(s->A[m], s->B[m], Si, H, d);
            double v[3];
            for (int k = 0; k < 3; ++k) { f0[k * n + i] = d[k]; v[k] = Si[k] + d[k] * dt; }
            const double L = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            nv[i] = L;
            for (int k = 0; k < 3; ++k) sp[k * n + i] = v[k] / L;
         }
         exch_only(s, sp, sp + n, sp + 2 * n, ex1, ex1 + n, ex1 + 2 * n);
         for (int i = 0; i < n; ++i) {
            const int m = s->type[i];
            const double Si[3] = {S[i], S[n + i], S[2 * n + i]};
            const double Sp[3] = {sp[i], sp[n + i], sp[2 * n + i]};
            double Ha[3], H1[3], f1[3], u[3];
            aniso_field(s, i, Sp, Ha);
            for (int k = 0; k < 3; ++k) H1[k] = ex1[k * n + i] + Ha[k] + Happ[k];
            f_eval(s->A[m], s->B[m], Sp, H1, f1);
            for (int k = 0; k < 3; ++k) u[k] = Si[k] + 0.5 * dt * (f0[k * n + i] + f1[k]);
            const double L = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
            const double s1[3] = {u[0] / L, u[1] / L, u[2] / L};
            const double l[3] = {lam[i], lam[n + i], lam[2 * n + i]};
            const double ls = l[0] * s1[0] + l[1] * s1[1] + l[2] * s1[2];
            double u_b[3], a1[3], sdir[3], hb[3];
            for (int k = 0; k < 3; ++k) { u_b[k] = (l[k] - ls * s1[k]) / L; a1[k] = 0.5 * dt * u_b[k]; }
            f_vjp(s->A[m], s->B[m], Sp, H1, a1, sdir, hb);
            for (int k = 0; k < 3; ++k) {
               ub[k * n + i] = u_b[k];
               spb[k * n + i] = sdir[k];
               Hb1[k * n + i] = hb[k];
               gH[k] += hb[k];
               gJ += hb[k] * ex1[k * n + i];
            }
            if (s->uniaxial) {
               const double e[3] = {s->kux[m], s->kuy[m], s->kuz[m]};
               const double he = hb[0] * e[0] + hb[1] * e[1] + hb[2] * e[2];
               const double se = Sp[0] * e[0] + Sp[1] * e[1] + Sp[2] * e[2];
               gK += 2.0 * he * se / s->mus_SI[m];
            }
         }
         /* s'bar += transposed exchange gather of H1bar + anisotropy */
         exch_transposed(s, Hb1, tmp, f1s);
         for (int i = 0; i < n; ++i) {
            const int m = s->type[i];
            const double Si[3] = {S[i], S[n + i], S[2 * n + i]};
            const double Sp[3] = {sp[i], sp[n + i], sp[2 * n + i]};
            double spbar[3], hb1[3] = {Hb1[i], Hb1[n + i], Hb1[2 * n + i]};
            for (int k = 0; k < 3; ++k) spbar[k] = spb[k * n + i] + tmp[k * n + i];
            if (s->uniaxial) {
               const double e[3] = {s->kux[m], s->kuy[m], s->kuz[m]};
               const double he = hb1[0] * e[0] + hb1[1] * e[1] + hb1[2] * e[2];
               for (int k = 0; k < 3; ++k) spbar[k] += 2.0 * s->ku2[m] * he * e[k];
            }
            if (s->cubic)
               for (int k = 0; k < 3; ++k) spbar[k] += 6.0 * s->kc4[m] * Sp[k] * Sp[k] * hb1[k];
            const double sps = spbar[0] * Sp[0] + spbar[1] * Sp[1] + spbar[2] * Sp[2];
            double vb[3], a0[3];
            for (int k = 0; k < 3; ++k) {
               vb[k] = (spbar[k] - sps * Sp[k]) / nv[i];
               a0[k] = 0.5 * dt * ub[k * n + i] + dt * vb[k];
            }
            double Ha[3], H0[3], sdir[3], hb[3];
            aniso_field(s, i, Si, Ha);
            for (int k = 0; k < 3; ++k) H0[k] = ex0[k * n + i] + Ha[k] + Happ[k];
            f_vjp(s->A[m], s->B[m], Si, H0, a0, sdir, hb);
            for (int k = 0; k < 3; ++k) {
               sb[k * n + i] = ub[k * n + i] + vb[k] + sdir[k];
               Hb0[k * n + i] = hb[k];
               gH[k] += hb[k];
               gJ += hb[k] * ex0[k * n + i];
            }
            if (s->uniaxial) {
               const double e[3] = {s->kux[m], s->kuy[m], s->kuz[m]};
               const double he = hb[0] * e[0] + hb[1] * e[1] + hb[2] * e[2];
               const double se = Si[0] * e[0] + Si[1] * e[1] + Si[2] * e[2];
               gK += 2.0 * he * se / s->mus_SI[m];
            }
         }
         exch_transposed(s, Hb0, tmp, f1s);
         for (int i = 0; i < n; ++i) {
            const int m = s->type[i];
            const double Si[3] = {S[i], S[n + i], S[2 * n + i]};
            double hb0[3] = {Hb0[i], Hb0[n + i], Hb0[2 * n + i]};
            for (int k = 0; k < 3; ++k) lam[k * n + i] = sb[k * n + i] + tmp[k * n + i];
            if (s->uniaxial) {
               const double e[3] = {s->kux[m], s->kuy[m], s->kuz[m]};
               const double he = hb0[0] * e[0] + hb0[1] * e[1] + hb0[2] * e[2];
               for (int k = 0; k < 3; ++k) lam[k * n + i] += 2.0 * s->ku2[m] * he * e[k];
            }
            if (s->cubic)
               for (int k = 0; k < 3; ++k) lam[k * n + i] += 6.0 * s->kc4[m] * Si[k] * Si[k] * hb0[k];
            if (t >= 1) lam[2 * n + i] += 2.0 * w * (mz[t] - target[t - 1]) * s->mus[m] / musum;
         }
      }
   }
   grad[0] = gJ; grad[1] = gK; grad[2] = gH[0]; grad[3] = gH[1]; grad[4] = gH[2];
   free(cp); free(seg); free(mz); free(work); free(cur); free(lam); free(ex0); free(ex1); free(sp);
   free(Hb1); free(Hb0); free(tmp); free(spb); free(sb); free(ub); free(f0); free(nv); free(f1s);
   return loss;
}

/* loss of the forward trajectory only (for finite differences) */
double vref_trajectory_loss(const vref_sys* s, const double* sx0, const double* sy0, const double* sz0,
                            int64_t nsteps, const double* target, double w) {
   const int n = s->n;
   double musum = 0.0;
   for (int i = 0; i < n; ++i) musum += s->mus[s->type[i]];
   double* cur = (double*)malloc(sizeof(double) * 3 * n);
   double* work = (double*)malloc(sizeof(double) * 15 * n);
   memcpy(cur, sx0, sizeof(double) * n);
   memcpy(cur + n, sy0, sizeof(double) * n);
   memcpy(cur + 2 * n, sz0, sizeof(double) * n);
   double loss = 0.0;
   for (int64_t t = 0; t < nsteps; ++t) {
      vref_llg_heun_step(s, cur, cur + n, cur + 2 * n, NULL, work);
      double m = 0.0;
      for (int i = 0; i < n; ++i) m += s->mus[s->type[i]] * cur[2 * n + i];
      const double r = m / musum - target[t];
      loss += w * r * r;
   }
   free(cur);
   free(work);
   return loss;
}

/* m_z(t) for t = 1..nsteps (targets) */
void vref_mz_trajectory(const vref_sys* s, const double* sx0, const double* sy0, const double* sz0,
                        int64_t nsteps, double* mz_out) {
   const int n = s->n;
   double musum = 0.0;
   for (int i = 0; i < n; ++i) musum += s->mus[s->type[i]];
   double* cur = (double*)malloc(sizeof(double) * 3 * n);
   double* work = (double*)malloc(sizeof(double) * 15 * n);
   memcpy(cur, sx0, sizeof(double) * n);
   memcpy(cur + n, sy0, sizeof(double) * n);
   memcpy(cur + 2 * n, sz0, sizeof(double) * n);
   for (int64_t t = 0; t < nsteps; ++t) {
      vref_llg_heun_step(s, cur, cur + n, cur + 2 * n, NULL, work);
      double m = 0.0;
      for (int i = 0; i < n; ++i) m += s->mus[s->type[i]] * cur[2 * n + i];
      mz_out[t] = m / musum;
   }
   free(cur);
   free(work);
}

/* magnetization_statistic_t::calculate_magnetization
 * (src/statistics/magnetization.cpp:134-180): per mask bin sum(mu s), sum(mu),
 * normalised to (m_hat, |m|/m_sat); empty bins zeroed.  out: 4*mask_size. */
void vref_magnetization(int n, const int* mask, int mask_size, const double* sx, const double* sy,
                        const double* sz, const double* mm, double* out) {
   memset(out, 0, sizeof(double) * 4 * mask_size);
   for (int atom = 0; atom < n; ++atom) {
      const int id = mask[atom];
      out[4 * id + 0] += sx[atom] * mm[atom];
      out[4 * id + 1] += sy[atom] * mm[atom];
      out[4 * id + 2] += sz[atom] * mm[atom];
      out[4 * id + 3] += mm[atom];
   }
   for (int id = 0; id < mask_size; ++id) {
      const double msat = out[4 * id + 3];
      const double magm = sqrt(out[4 * id + 0] * out[4 * id + 0] + out[4 * id + 1] * out[4 * id + 1] +
                               out[4 * id + 2] * out[4 * id + 2]);
      if (msat == 0.0) {  /* zero_list: empty bins */
         out[4 * id + 0] = out[4 * id + 1] = out[4 * id + 2] = out[4 * id + 3] = 0.0;
         continue;
      }
      out[4 * id + 0] /= magm;
      out[4 * id + 1] /= magm;
      out[4 * id + 2] /= magm;
      out[4 * id + 3] = magm / msat;
   }
}

/* energy_statistic_t::calculate (src/statistics/energy.cpp:141-258): per mask
 * bin, sums of mu * E over atoms; exchange and magnetostatic halved.
 * out: 5*mask_size as [total | exchange | anisotropy | applied | magnetostatic]. */
void vref_energy(const vref_sys* s, const int* mask, int mask_size, const double* sx,
                 const double* sy, const double* sz, const double* mm, double* out) {
   double* tot = out;
   double* exc = out + mask_size;
   double* ani = out + 2 * mask_size;
   double* app = out + 3 * mask_size;
   double* mst = out + 4 * mask_size;
   memset(out, 0, sizeof(double) * 5 * mask_size);
   for (int atom = 0; atom < s->n; ++atom) {
      double e[4];
      vref_spin_energy(s, sx, sy, sz, atom, sx[atom], sy[atom], sz[atom], e);
      const int id = mask[atom];
      exc[id] += e[0] * mm[atom];
      ani[id] += e[1] * mm[atom];
      app[id] += e[2] * mm[atom];
      mst[id] += e[3] * mm[atom];
   }
   for (int id = 0; id < mask_size; ++id) {
      exc[id] *= 0.5;
      mst[id] *= 0.5;
      tot[id] = exc[id] + ani[id] + app[id] + mst[id];
   }
}
