/*
 * gasatt_oracle.h - CPU FP64 oracle for the PIC-MCC electron step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * algorithm (its CUDA kernels and MATLAB functions), used by tests/, by the
 * smoke check and by bench.py's CPU baseline leg as the checker.  The product
 * (libgasatt) never links, loads or calls it.
 *
 * Every function cites the reference file:line it restates.  The quirk flags
 * (GASATT_Q_*, include/gasatt.h) select between reproducing a reference
 * behaviour and its corrected form.
 */
#ifndef GASATT_ORACLE_H
#define GASATT_ORACLE_H

#include <stdint.h>
#include "../include/gasatt.h"

#ifdef __cplusplus
extern "C" {
#endif

void orc_set_threads(int n);
int  orc_get_threads(void);

/* ---- counter-based RNG (Philox4x32-10, Salmon et al. SC'11) ---- */
void   orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double orc_u01(uint32_t hi, uint32_t lo);           /* (0,1) from 52 bits */
uint64_t orc_child_id(uint64_t parent, int64_t step);

/* ---- MATLAB built-ins restated ---- */
double orc_interp1(const double *x, int sx, const double *y, int sy, int n, double xq);

/* ---- find_CS0.m ---- */
void orc_find_cs0(const gasatt_tables *t, const double *E_keV, int64_t n,
                  double *s_el, double *s_ion, double *s_exc, unsigned flags);
/* electron_collision.m:12-33 : xInterp[ne], yInterp[ne], V_interp[181*ne]; returns ne or <0 */
int orc_elastic_tables(const gasatt_tables *t, double *xInterp, double *yInterp, double *V_interp);

/* ---- kernels of the reference, one call = one launch ---- */
void orc_em2(double *x, double *y, double *z, double *vx, double *vy, double *vz,
             double *r, double *phi, double *vr, int *del, int64_t n,
             double Rp, double Lp, double PHIp, double dt, unsigned flags);
void orc_em7(const double *r, const double *z, const double *q, const double *vr,
             const double *vz, double *jr, double *jz, const int *del, int64_t n,
             int nr, int nz, double dr, double dz, double FN, double PHIp);
void orc_em3_1(double *Er, double *Ez, double *H, int nr, int nz,
               double mu, double dr, double dz, double dt);
void orc_em3(const double *Er0, const double *Ez0, const double *H0, double *Er, double *Ez,
             const double *jr, const double *jz, int nr, int nz,
             double eps, double dr, double dz, double dt, unsigned flags);
void orc_em4(double *x, double *y, double *z, double *vx, double *vy, double *vz,
             double *r, double *phi, const double *vr, const double *Er, const double *Ez,
             const double *H, const double *q, const double *m, double *E, int *del,
             int64_t n, double Rp, double Lp, double PHIp, int nr, int nz,
             double mu, double c, double dr, double dz, double dt, unsigned flags);
/* electron_transport.cu:3-229 with injected draws (n x GASATT_MCC_NDRAW) */
void orc_electron_transport(double *x, double *y, double *z, double *vx, double *vy, double *vz,
                            const double *sig_el, const double *sig_ion, const double *sig_exc,
                            const double *energy, const double *xInterp, const double *yInterp,
                            const double *V_interp, int ne,
                            const double *density, const double *temperature, int64_t ncell,
                            const double *dphi, const double *t_exc, int n_exc,
                            uint8_t *sec, double *svx, double *svy, double *svz,
                            double *sample_out, double *ivx, double *ivy, double *ivz,
                            const int *sum_cell0, int rmax, int cellnumxy,
                            double dr, double dz, double dt, int64_t n,
                            const double *draws, unsigned flags);

/* ---- MATLAB drop-ins ---- */
/* REBOND.m:1-70.  pos, vel: n x 3 column-major (leading dimensions ldp, ldv),
 * updated in place; returns N_boundary, or -1 when a particle needs more than
 * max_wraps wedge wraps. */
int64_t orc_rebond(double *pos, int64_t ldp, const double *r, const double *phi, double *vel,
                   int64_t ldv, int64_t n, double Lp, double PHIp, int max_wraps);
void orc_free_motion(const double *vx, const double *vy, const double *vz,
                     const double *x, const double *y, const double *z, int64_t n, double dt,
                     double *xn, double *yn, double *zn, double *rn, double *phin);
void orc_particle_density(double dr, double dz, const double *dphi, int rmax,
                          const double *r, const double *phi, const double *z, int64_t n,
                          int cellnumxy, const double *sum_cell, const double *VC,
                          int64_t ncell, double FN, double *density);
/* species arrays n x 3 column-major; see gasatt_electricmagneticfield6 */
int orc_electricmagneticfield6(double *e_pos, double *e_vel, int64_t n_e,
                               double *i1_pos, double *i1_vel, int64_t n_i1,
                               double *i2_pos, double *i2_vel, int64_t n_i2,
                               double *Er, double *Ez, double *H, int nr, int nz,
                               double delta, double dt, double Rp, double Lp,
                               double PHIp, double FN, int cycle_time, double *kin,
                               int64_t *n_e_out, int64_t *n_i1_out, int64_t *n_i2_out,
                               unsigned flags);
int orc_electron_collision(double *e_pos, double *e_vel, int64_t n_e, int64_t cap_e,
                           double *i1_pos, double *i1_vel, int64_t n_i1, int64_t cap_i1,
                           const gasatt_tables *tab, const double *kin,
                           const double *sum_cell, int rmax, int cellnumxy,
                           const double *density, const double *temperature, int64_t ncell,
                           double PHIp, const double *phimax, double dr, double dz,
                           const double *sig_el, const double *sig_ion, const double *sig_exc,
                           double dt, const double *draws,
                           int64_t *n_e_out, int64_t *n_i1_out, unsigned flags);

/* ---- resident step, corrected physics (Cartesian u = gamma v form) ---- */
typedef struct orc_xs {
  int G;  double lnEmin, dlnE;        /* log grid */
  double *sig_el, *sig_ion, *sig_exc; /* [G], m^2 */
  double *cdf;                        /* [G*181] normalised elastic CDF */
  double *edep;                       /* [G] mean excitation energy loss [eV] */
  double exc_kmin;                    /* lowest excitation threshold [eV] */
  double nu_max;                      /* s^-1, FP64 bound */
  double exc_k[16], exc_A[16], exc_om[16], exc_nu[16], exc_ga[16]; int n_exc;
} orc_xs;
orc_xs *orc_xs_create(const gasatt_tables *t, int G, double emin_ev, double emax_ev,
                      double n_gas, double c, double me, double qe);
void orc_xs_free(orc_xs *xs);
double orc_xs_nu_max(const orc_xs *xs);
/* 0 sig_el, 1 sig_ion, 2 sig_exc, 4 edep (length G), 3 cdf (G x 181) */
const double *orc_xs_array(const orc_xs *xs, int which);

typedef struct orc_counters {
  int64_t ion, ela, exc, nul, lost, cap_overflow;
  int64_t exc_loss_fx;                /* excitation losses, sum of llrint(E_dep * 2^16) [eV] */
} orc_counters;

/* N2+ ion store of the resident step (Cartesian u = gamma v form).  Ions are
 * born one per ionization (electron_transport.cu:202-204) when the store is
 * given, at the parent's position with a Maxwellian velocity at
 * cfg->gas_temperature, id = the secondary electron's id, charge number 1. */
typedef struct orc_ions {
  double *x, *y, *z, *ux, *uy, *uz;
  uint64_t *id;
  uint8_t *alive;
  int8_t *q;
  int64_t n, cap;
  int64_t overflow, lost;
} orc_ions;

/* one particle pass of step s: gather + kick + half drift + half drift +
 * deposit, then the null-collision MCC at the end of the step (an ionization
 * appends its secondary at the parent's position).  Arrays x..alive have
 * capacity cap; *n grows with births.  jr/jz receive the current density
 * [A/m^2] (overwritten).  gas: per-cell N2 density (n_r x n_z, column-major,
 * cell ir = floor(r/dr), iz = floor(z/dz), both clamped to the grid) or NULL
 * for cfg->gas_density everywhere; xs->nu_max must bound the largest density.
 * gas_T: per-cell temperature [K] for the newborn ions (same layout), or NULL
 * for cfg->gas_temperature. */
int orc_sim_pass(const gasatt_sim_config *cfg, const orc_xs *xs, int64_t step,
                 double *x, double *y, double *z, double *ux, double *uy, double *uz,
                 uint64_t *id, uint8_t *alive, int64_t *n, int64_t cap,
                 const double *Er, const double *Ez, const double *H,
                 double *jr, double *jz, int do_kick, int do_mcc, const double *gas,
                 const double *gas_T, orc_ions *ions, orc_counters *cnt);
/* ion push over dt_i = cfg->ion_subcycle * cfg->dt: gather, Boris kick with
 * charge q e and mass cfg->m_ion, two half drifts (absorbed beyond Rp,
 * reflected at the z ends), deposit of the ion current density [A/m^2] into
 * jr/jz (overwritten); the field update adds it to the electrons' until the
 * next ion push. */
void orc_ion_push(const gasatt_sim_config *cfg, orc_ions *ions, const double *Er,
                  const double *Ez, const double *H, double *jr, double *jz);
/* field sub-cycle: H(-dt/4), [H(dt/2), E(dt/2)] x 2 ratio, H(dt/4), dt = cfg->dt/ratio */
void orc_sim_fdtd(const gasatt_sim_config *cfg, double *Er, double *Ez, double *H,
                  const double *jr, const double *jz);
double orc_field_energy(const gasatt_sim_config *cfg, const double *Er, const double *Ez,
                        const double *H);

/* The reference's MATLAB CPU path, one call of electricmagneticfield3.m:111-319
 * for electrons (charge -e, mass m_e of that file): half drift, deletion
 * beyond the wall and the wedge/z rules (REBOND), nearest-cell current
 * (ind2vec), the field update in two halves, interp2 gather, explicit
 * relativistic kick, second half drift with the same rules.  Particles are
 * (x, y, z) and v (not gamma v); deleted ones get alive = 0 instead of being
 * removed.  Grids dense column-major: Er n_r x (n_z+1), Ez (n_r+1) x n_z,
 * H n_r x n_z; jr, jz (n_r x n_z) receive the step's current density.
 * delta: cell size, dt: particle step, PHIp: wedge angle, W: particles per
 * macro-particle.  Returns the electrons alive afterwards. */
int64_t orc_mcpu_step(int64_t n, double *x, double *y, double *z, double *vx, double *vy,
                      double *vz, uint8_t *alive, double *Er, double *Ez, double *H, double *jr,
                      double *jz, int nr, int nz, double delta, double dt, double PHIp, double W);

#ifdef __cplusplus
}
#endif
#endif
