/*
 * gasatt.h - C ABI of the B200 PIC-MCC electron step for the N2 X-ray gas
 * attenuator (axisymmetric r-z, Yee FDTD, null-collision Monte Carlo).
 *
 * Two groups of entry points:
 *
 *  1. Drop-ins for the MATLAB functions of the reference driver.  Each takes
 *     DEVICE pointers to column-major (MATLAB layout) arrays plus sizes and a
 *     context, and replaces one reference function:
 *        gasatt_find_CS0               find_CS0.m:1-61
 *        gasatt_free_motion            free_motion.m:1-9
 *        gasatt_particle_density       particle_density.m:1-38
 *        gasatt_electricmagneticfield6 electricmagneticfield6.m:1-188
 *                                      (EM2.cu, EM7.cu, EM3_1.cu, EM3.cu, EM4.cu)
 *        gasatt_electron_collision     electron_collision.m:1-75
 *                                      (electron_transport.cu:3-229)
 *     The cross-section tables are passed as HOST pointers in the shapes that
 *     MATLAB's readtable produces (see gasatt_tables below).
 *
 *  2. The resident simulation ("sim"): particles live in HBM in the
 *     library's own SoA layout (plain FP64 or FP32 split precision) and one
 *     call advances N steps of push + MCC + deposit + FDTD.
 *
 * Every function returns a gasatt status (0 = OK).  gasatt_last_error()
 * gives the message of the last failure on a context.  A context is used by
 * one host thread at a time; different contexts are independent.
 */
#ifndef GASATT_H
#define GASATT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define GASATT_OK            0
#define GASATT_E_ARG         1   /* bad argument / shape                     */
#define GASATT_E_CUDA        2   /* CUDA runtime error                       */
#define GASATT_E_CAPACITY    3   /* particle capacity exceeded               */
#define GASATT_E_NAN         4   /* non-finite value detected in a kernel    */
#define GASATT_E_TABLES      5   /* cross-section tables missing / invalid   */
#define GASATT_E_STATE       6   /* call out of order                        */
#define GASATT_E_NODEVICE    7   /* no CUDA device / library built without   */

/* ---------------------------------------------------------- quirk flags
 * Each bit reproduces one behaviour of the reference that the resident
 * simulation corrects.  The drop-ins default to GASATT_FAITHFUL (reference
 * behaviour); the simulation uses 0.
 */
#define GASATT_Q_EULER_KICK     (1u << 0)  /* EM4.cu:134-138 explicit kick, not Boris        */
#define GASATT_Q_ATAN_PHI       (1u << 1)  /* EM2.cu:30, EM4.cu:151 phi=atan(y/x) (axis mirror)*/
#define GASATT_Q_ER_END_COPY    (1u << 2)  /* EM3.cu:21-27 Er(z=0,Lp) copied, not PEC zero      */
#define GASATT_Q_EZ_AXIS_JSIGN  (1u << 3)  /* EM3.cu:35 axis Ez adds +jz                         */
#define GASATT_Q_EZ_RSHIFT      (1u << 4)  /* EM3.cu:39 radius (nr+1)dr at Ez node nr            */
#define GASATT_Q_XS_LINEAR_E    (1u << 5)  /* electron_transport.cu:89 keV compared to log(E)     */
#define GASATT_Q_COLL_LINEAR_P  (1u << 6)  /* electron_transport.cu:74-79 p=v dt n sigma         */
#define GASATT_Q_SEC_LAB_FRAME  (1u << 7)  /* electron_transport.cu:198-200 secondary about lab z */
#define GASATT_Q_EXC_POWF       (1u << 8)  /* electron_transport.cu:214-215 single-precision pow  */
#define GASATT_Q_XS_NAN         (1u << 9)  /* find_CS0.m:16-56 NaN/neg. outside the tables        */
#define GASATT_Q_PI7            (1u << 10) /* electron_transport.cu:53 pi = 3.1415926             */
#define GASATT_Q_CDF_NEXTBIN    (1u << 11) /* electron_transport.cu:103-121 rectangle CDF, next-bin inverse */
#define GASATT_FAITHFUL         0x0FFFu
/* input-convention bit for gasatt_electricmagneticfield6: positions arrive as
 * (r, phi, z) columns (electricmagneticfield6.m:113-115) instead of (x, y, z) */
#define GASATT_POS_IN_CYL       (1u << 16)

/* ------------------------------------------------ reference constants
 * The reference uses different values per file; the drop-ins use the value of
 * the file they replace.
 */
#define GASATT_EM_E        1.6e-19          /* electricmagneticfield6.m:11 */
#define GASATT_EM_ME       9.1096e-31       /* electricmagneticfield6.m:5  */
#define GASATT_EM_MION     4.65e-26         /* electricmagneticfield6.m:6-7 */
#define GASATT_EM_C        3e8              /* electricmagneticfield6.m:8  */
#define GASATT_EM_EPS      8.854187817e-12  /* electricmagneticfield6.m:9  */
#define GASATT_PI          3.141592653589793
#define GASATT_EM_MU       (4.0 * GASATT_PI * 1e-7) /* electricmagneticfield6.m:10 */
#define GASATT_MCC_E       1.6022e-19       /* electron_transport.cu:47 */
#define GASATT_MCC_C       3e8              /* electron_transport.cu:48 */
#define GASATT_MCC_ME      9.109e-31        /* electron_transport.cu:49 */
#define GASATT_MCC_MION    4.65e-26         /* electron_transport.cu:50 */
#define GASATT_MCC_KB      1.38064853e-23   /* electron_transport.cu:51 */
#define GASATT_MCC_PI7     3.1415926        /* electron_transport.cu:53 */
#define GASATT_MCC_Q0      6.514e-14        /* electron_transport.cu:208 */
#define GASATT_ION_I_EV    15.6             /* electron_transport.cu:60 */
#define GASATT_CS_Q0       6.542e-14        /* find_CS0.m:42 */
#define GASATT_A0SQ        2.8002852e-21    /* find_CS0.m:17, electron_collision.m:12 */

/* injected random draws per particle for gasatt_electron_collision:
 * [0] p1  [1] p2  [2] elastic angle / ionization split  [3] azimuth
 * [4..6] three standard normals (ion Maxwellian), used as float like curand_normal */
#define GASATT_MCC_NDRAW   8

/* --------------------------------------------------------------- tables
 * Raw N2 tables as MATLAB readtable gives them (electron_transport_field3.m:8-37),
 * column-major, HOST memory:
 *   t_el    2 x n_el      row 0 energy [keV], row 1 sigma [a0^2 per N atom]
 *   t_sel   n_sel x 2     energy [eV], sigma [1e-20 m^2]          (1..50 eV)
 *   t_sel_1 n_sel1 x 2    energy [eV], sigma [1e-20 m^2]          (5..50 eV)
 *   t_del   181+1 x n_del row 0 energies [keV], col 0 angles, DCS body
 *   t_sdel  181+1 x n_sdel same, low-energy DCS
 *   t_ion   n_ion x 2     energy [eV], sigma [1e-20 m^2]
 *   t_exc   n_exc x 5     k [eV], A, omega, nu, gamma
 */
typedef struct gasatt_tables {
  const double *t_el;    int n_el;
  const double *t_sel;   int n_sel;
  const double *t_sel_1; int n_sel1;
  const double *t_del;   int del_rows;  int del_cols;
  const double *t_sdel;  int sdel_rows; int sdel_cols;
  const double *t_ion;   int n_ion;
  const double *t_exc;   int n_exc;
} gasatt_tables;

/* -------------------------------------------------------------- context */
typedef struct gasatt_ctx gasatt_ctx;

int         gasatt_create(gasatt_ctx **ctx, int device, uint64_t seed);
int         gasatt_destroy(gasatt_ctx *ctx);
const char *gasatt_last_error(const gasatt_ctx *ctx);
/* stream (cudaStream_t as void*) used for every launch on this context; NULL = legacy default */
int         gasatt_set_stream(gasatt_ctx *ctx, void *stream);
int         gasatt_synchronize(gasatt_ctx *ctx);
/* number of kernels this context launched since creation (monotone counter) */
int64_t     gasatt_kernel_launches(const gasatt_ctx *ctx);
const char *gasatt_version(void);

/* ------------------------------------------------------------- drop-ins */

/* find_CS0.m:1-61.  E_keV, sig_* : device, length n.  Tables: host. */
int gasatt_find_CS0(gasatt_ctx *ctx, const gasatt_tables *tab,
                    const double *E_keV, int64_t n,
                    double *sig_el, double *sig_ion, double *sig_exc,
                    unsigned flags);

/* free_motion.m:1-9.  All device arrays of length n. */
int gasatt_free_motion(gasatt_ctx *ctx,
                       const double *vx, const double *vy, const double *vz,
                       const double *x, const double *y, const double *z,
                       int64_t n, double dt,
                       double *xn, double *yn, double *zn, double *rn, double *phin);

/* REBOND.m:1-70: the boundary rule of the reference's gpuArray drivers.
 * pos, vel: device, n x 3 column-major with leading dimensions ld_pos, ld_vel
 * (x, y, z and vx, vy, vz), updated in place; r, phi: device, length n (the
 * particles' radius and azimuth).  An azimuth outside [0, PHIp] is wrapped
 * into it one wedge at a time, turning (vx, vy) by the wedge angle each time,
 * and x, y are rebuilt from r and the new azimuth; then z is reflected at Lp
 * and at 0 (vz flipped).  *n_boundary: wraps plus reflections.  An azimuth
 * more than 4096 wedges outside fails with GASATT_E_ARG (the reference would
 * loop on). */
int gasatt_rebond(gasatt_ctx *ctx, double *pos, int64_t ld_pos, const double *r,
                  const double *phi, double *vel, int64_t ld_vel, int64_t n, double Lp,
                  double PHIp, int64_t *n_boundary);

/* particle_density.m:1-38 (10-argument form).
 * dphi, sum_cell: device arrays of length rmax (sum_cell(k) = cells with r index <= k).
 * r, phi, z: device, length n.  VC: device, length cellnumxy (volume of the
 * cells of one z layer, calculate_VC.m).  density: device, length ncell
 * (= cellnumxy * zmax), overwritten.  Particles whose cell index falls
 * outside [1, ncell] are not counted. */
int gasatt_particle_density(gasatt_ctx *ctx, double dr, double dz,
                            const double *dphi, int rmax,
                            const double *r, const double *phi, const double *z,
                            int64_t n, int cellnumxy, const double *sum_cell,
                            const double *VC, int64_t ncell, double FN,
                            double *density);

/* gasatt_particle_density without any device allocation.  It has no
 * counterpart in the reference: it exists for callers that must not call
 * cudaMalloc/cudaFree themselves or through this library -- above all a MEX
 * gateway running inside MATLAB, whose gpuArray memory pool owns the device
 * memory (a private allocation competes with that pool, and cudaFree stalls
 * the whole device).  gasatt_particle_density takes its per-cell counts from
 * the context's scratch buffer, which it may grow with cudaMalloc; this call
 * counts instead into a fixed array compiled into the library, of
 * GASATT_DENSITY_NOALLOC_MAX_CELLS 64-bit counters (8 MiB, held by every
 * device that loads the library until the process exits).
 *  - Arguments and result are those of gasatt_particle_density.
 *  - ncell > GASATT_DENSITY_NOALLOC_MAX_CELLS is rejected with
 *    GASATT_E_CAPACITY (nothing is launched).
 *  - Every call looks up the array's device address on the context's device
 *    (cudaGetSymbolAddress), so the call stays valid after that device's
 *    context is reset (the array then starts over, zeroed).  The first call
 *    on a device also loads the library's device code there; make that first
 *    call before any stream capture.
 *  - The counters are zeroed on the context's stream at the start of every
 *    call.  All calls on a device share the one array, so calls whose work
 *    overlaps on the GPU (other streams, other contexts, other host threads)
 *    race and give wrong densities; keep them ordered. */
#define GASATT_DENSITY_NOALLOC_MAX_CELLS (1 << 20)
int gasatt_particle_density_noalloc(gasatt_ctx *ctx, double dr, double dz,
                                    const double *dphi, int rmax,
                                    const double *r, const double *phi, const double *z,
                                    int64_t n, int cellnumxy, const double *sum_cell,
                                    const double *VC, int64_t ncell, double FN,
                                    double *density);

/* electricmagneticfield6.m:1-188.  Species arrays are device, column-major
 * with leading dimension equal to their count (n x 3).  Positions arrive as
 * (r,phi,z) when GASATT_POS_IN_CYL is set (the reference convention) else
 * (x,y,z); they leave as (x,y,z).  Deleted particles (r > Rp) are removed in
 * place, order kept; the new counts are returned in *_out and the first
 * n_out rows of each array (leading dimension unchanged) hold the survivors.
 * Er: n_r x (n_z+1), Ez: (n_r+1) x n_z, Hphi: n_r x n_z, updated in place.
 * electron_kinetic: device, length n_e, kinetic energy [keV] of the surviving
 * electrons.  cycle_time/5 particle steps of 5*dt are taken
 * (electricmagneticfield6.m:134-138). */
int gasatt_electricmagneticfield6(gasatt_ctx *ctx,
                                  double *e_pos, double *e_vel, int64_t n_e,
                                  double *i1_pos, double *i1_vel, int64_t n_i1,
                                  double *i2_pos, double *i2_vel, int64_t n_i2,
                                  double *Er, double *Ez, double *Hphi,
                                  int n_r, int n_z,
                                  double delta, double dt, double Rp, double Lp,
                                  double PHIp, double FN, int cycle_time,
                                  double *electron_kinetic,
                                  int64_t *n_e_out, int64_t *n_i1_out, int64_t *n_i2_out,
                                  unsigned flags);

/* electron_collision.m:1-75 with electron_transport.cu:3-229.
 * e_pos/e_vel: device, column-major with leading dimension cap_e (>= n_e plus
 * room for one secondary per electron); i1_pos/i1_vel likewise with cap_i1.
 * electron_kinetic, sig_*: device length n_e.  density, temperature: device,
 * length ncell.  sum_cell, phimax: host, length rmax.  draws: optional device
 * array n_e x GASATT_MCC_NDRAW (row-major per particle) of injected draws;
 * NULL draws from Philox keyed on (context seed, particle index, call count).
 * Secondaries are appended to the electrons and ions to ion1 in parent order
 * (MATLAB logical indexing, electron_collision.m:63-75). */
int gasatt_electron_collision(gasatt_ctx *ctx,
                              double *e_pos, double *e_vel, int64_t n_e, int64_t cap_e,
                              double *i1_pos, double *i1_vel, int64_t n_i1, int64_t cap_i1,
                              const gasatt_tables *tab,
                              const double *electron_kinetic,
                              const double *sum_cell, int rmax, int cellnumxy,
                              const double *density, const double *temperature, int64_t ncell,
                              double PHIp, const double *phimax, double dr, double dz,
                              const double *sig_el, const double *sig_ion, const double *sig_exc,
                              double dt_transport, const double *draws,
                              int64_t *n_e_out, int64_t *n_i1_out, unsigned flags);

/* ------------------------------------------------------ resident simulation */
#define GASATT_FP64        0   /* plain FP64: r, z, u_r, u_theta, u_z (+ id)       */
#define GASATT_FP32_SPLIT  1   /* int32 cell key + FP32 offsets + FP32 u (+ id)    */

typedef struct gasatt_sim_config {
  int      n_r, n_z;        /* cells; Er n_r x (n_z+1), Ez (n_r+1) x n_z, Hphi n_r x n_z */
  double   dr, dz;          /* cell size [m] */
  double   dt;              /* particle step [s] */
  int      fdtd_ratio;      /* field sub-cycle: 2*ratio half-updates of dt/2 each per ratio*dt of
                               particle time; the product uses 1 (electricmagneticfield6.m:134-151 uses 5) */
  double   PHIp;            /* azimuthal extent of a macro-particle shell [rad] (2*pi: full ring) */
  double   FN;              /* real electrons per macro-particle */
  double   gas_density;     /* N2 number density [m^-3] */
  double   gas_temperature; /* [K] */
  double   q_e, m_e, c, eps0, mu0, kb, m_ion;  /* constants (SI); q_e > 0 */
  int      precision;       /* GASATT_FP64 / GASATT_FP32_SPLIT */
  int64_t  capacity;        /* max electrons */
  int64_t  ion_capacity;    /* N2+ ions stored at most (0: no ion species; ionizations are
                               only counted).  One ion per ionization, born at the parent's
                               position with a Maxwellian velocity at gas_temperature
                               (electron_transport.cu:202-204), pushed in the same fields
                               every ion_subcycle steps, its current added to the electrons' */
  uint64_t seed;
  unsigned flags;           /* quirk flags (0 for the product) */
  int      sort_period;     /* steps between cell re-sorts (0 = never) */
  int      secondaries;     /* 1: ionization births enabled */
  int      table_n;         /* log-energy grid points (2048) */
  double   table_emin_ev, table_emax_ev;  /* 0.1 eV, 30 keV */
  int      ion_subcycle;    /* electron steps per ion push (50); the ion step is ion_subcycle*dt */
  /* launch-shape knobs (results do not depend on them; 0 = the default, and
   * the autotuner of the Python package picks them per workload): */
  int      fdtd_tile_rows;  /* rows of the field update's per-warp patch: 12, 16 or 20
                               (output 26 columns x rows - 6 per patch); default 12 */
  int      pass_chunk;      /* FP32 particle pass: particles per chunk a block takes,
                               a multiple of 256 (256..1792); default 1792 */
  int      gather;          /* FP32 form, how the push reads E and H: 1 = packed 2 x 2
                               quads the field update writes beside the fields (three
                               16-byte loads per electron, 48 more bytes written per
                               cell), 2 = the four corners straight from the fields;
                               0 = quads when the capacity is at least 4 electrons per
                               cell.  Both give the same bits. */
} gasatt_sim_config;

typedef struct gasatt_diag {
  int64_t n_alive;          /* electrons alive */
  int64_t n_total;          /* slots in use (alive + dead not yet compacted) */
  int64_t n_ionizations;    /* cumulative ionization events (= secondaries born) */
  int64_t n_elastic, n_excitation, n_null;   /* cumulative collision branches */
  int64_t n_lost_wall;      /* cumulative electrons absorbed at r = Rp */
  int64_t n_ions;           /* ions alive in the store (ion_capacity > 0) */
  double  kinetic_ev;       /* sum of electron kinetic energy [eV] (x FN not applied) */
  double  field_energy_j;   /* electromagnetic field energy [J] */
  int64_t steps;            /* steps taken */
  int32_t status_flags;     /* bit0 NaN seen, bit1 capacity overflow, bit2 ion capacity overflow,
                               bit3 a bounded device wait gave up (field-update tile copy or
                               sort scan): the results since are not to be trusted */
  int64_t n_ion_lost_wall;  /* cumulative ions absorbed at r = Rp */
  double  ion_kinetic_ev;   /* sum of ion kinetic energy [eV] (x FN not applied) */
  double  net_charge_c;     /* charge of the macro-particles in the domain [C]:
                               q_e FN (sum of ion charge numbers - electrons alive) */
  double  collision_loss_ev;/* cumulative electron energy given to the gas [eV] (x FN not
                               applied): 15.6 eV per ionization + the excitation losses */
  double  wall_loss_ev;     /* cumulative kinetic energy of the electrons and ions absorbed
                               at r = Rp [eV] (x FN not applied) */
} gasatt_diag;

typedef struct gasatt_sim gasatt_sim;

int gasatt_sim_default_config(gasatt_sim_config *cfg);
int gasatt_sim_create(gasatt_ctx *ctx, const gasatt_sim_config *cfg,
                      const gasatt_tables *tab, gasatt_sim **sim);
int gasatt_sim_destroy(gasatt_sim *sim);
/* the configuration the simulation was created with (sizes for a caller that
 * allocates the arrays of gasatt_sim_get_fields and the like) */
int gasatt_sim_get_config(const gasatt_sim *sim, gasatt_sim_config *cfg);
/* particle state in SI, axisymmetric frame: r, z [m]; u = gamma*v [m/s] in
 * (r, theta, z); id: 64-bit identity keying the random stream.
 * on_device: 1 = pointers are device memory, 0 = host memory. */
int gasatt_sim_load(gasatt_sim *sim, const double *r, const double *z,
                    const double *ur, const double *ut, const double *uz,
                    const uint64_t *id, int64_t n, int on_device);
/* Photoionization births generated on the device, replacing the particles
 * like gasatt_sim_load (INCIDENCE1.m:51-158 draws the reference's births on
 * the host): each of n_photo photons of photon_keV gives a photoelectron
 * (photon energy minus the N K-shell binding, 410 eV; direction density
 * ~ (d . x)^2 about the polarisation x) and an isotropic 360 eV Auger
 * electron, both at a Rayleigh(sigma_r) radius (clipped inside the wall),
 * uniform azimuth and uniform z.  Philox draws keyed on (seed, photon index).
 * Ids: id_base + 2k (photoelectron of photon k), id_base + 2k + 1 (Auger). */
int gasatt_sim_birth_photo(gasatt_sim *sim, int64_t n_photo, double photon_keV, double sigma_r,
                           uint64_t seed, uint64_t id_base);
/* Ion species (cfg->ion_capacity > 0).  load_ions replaces the ions (the
 * reference's ion1 and ion2 arrays of electricmagneticfield6.m:1, charge
 * numbers 1 and 2, mass cfg->m_ion, electricmagneticfield6.m:6-7,68-69); charge
 * NULL means all singly charged.  gasatt_sim_load and gasatt_sim_birth_photo
 * start a new run and clear the ions, so load ions after them.  read_ions
 * returns the ion slots in use (dead ions: r = -1), the same layout as
 * gasatt_sim_read.  Ions are FP64 in both precision forms. */
int gasatt_sim_load_ions(gasatt_sim *sim, const double *r, const double *z,
                         const double *ur, const double *ut, const double *uz,
                         const uint64_t *id, const int8_t *charge, int64_t n, int on_device);
int gasatt_sim_read_ions(gasatt_sim *sim, double *r, double *z, double *ur, double *ut,
                         double *uz, uint64_t *id, int8_t *charge, int64_t cap, int64_t *n,
                         int on_device);
/* Per-cell N2 density [m^-3] for the collisions: n_r x n_z values, column-major
 * (cell ir + n_r iz covers [ir dr, (ir+1) dr) x [iz dz, (iz+1) dz)); NULL goes
 * back to the uniform cfg->gas_density.  Replaces the density lookup by cell
 * of electron_transport.cu:64-76 (the reference's density_cells array, which
 * its DSMC neutral solver could fill) for the resident simulation: an electron
 * collides against the density of the cell it ends the step in, and the
 * null-collision bound becomes max(density) x max(sigma_tot v).  Values must be
 * finite and >= 0 (GASATT_E_ARG otherwise).  Collisions still queued are
 * applied first, with the old density; the step graphs are rebuilt, so a
 * batch (gasatt_batch_create) holding this simulation must be created after
 * the call.  on_device: 1 = device pointer, 0 = host pointer. */
int gasatt_sim_set_gas_density(gasatt_sim *sim, const double *density, int on_device);
/* Per-cell gas temperature [K] (n_r x n_z, column-major like the density;
 * NULL: the uniform cfg->gas_temperature): the temperature of the
 * reference's temperature_cells array, which its collision kernel reads for
 * the newborn ion's Maxwellian (electron_transport.cu:202-204).  An ion born
 * in a cell gets velocity components of spread sqrt(kb T / m_ion) of that
 * cell.  Values finite and >= 0.  Collisions still queued are applied first;
 * the step graphs are rebuilt, so create a batch after this call. */
int gasatt_sim_set_gas_temperature(gasatt_sim *sim, const double *temperature, int on_device);
int gasatt_sim_read(gasatt_sim *sim, double *r, double *z,
                    double *ur, double *ut, double *uz, uint64_t *id,
                    int64_t cap, int64_t *n, int on_device);
/* fields in the reference layout (column-major): Er n_r x (n_z+1), Ez (n_r+1) x n_z, Hphi n_r x n_z */
int gasatt_sim_set_fields(gasatt_sim *sim, const double *Er, const double *Ez,
                          const double *Hphi, int on_device);
int gasatt_sim_get_fields(gasatt_sim *sim, double *Er, double *Ez, double *Hphi,
                          int on_device);
/* current density [A/m^2] deposited by the last particle pass (n_r x n_z each) */
int gasatt_sim_get_current(gasatt_sim *sim, double *jr, double *jz, int on_device);
/* advance nsteps steps of FDTD + push + deposit + MCC (replayed from CUDA
 * graphs).  The collisions of a step are applied at its end; the library may
 * defer them into the next step's graph, and every call that observes the
 * particles (read, diag, counts, sort, run_host) applies them first. */
int gasatt_sim_step(gasatt_sim *sim, int nsteps);
/* cell re-sort + compaction of dead slots now */
int gasatt_sim_sort(gasatt_sim *sim);
int gasatt_sim_diag(gasatt_sim *sim, gasatt_diag *out);
/* End-to-end entry with HOST buffers (the call a MATLAB host makes):
 * pos/vel are n x 3 column-major Cartesian arrays in SI (leading dimension
 * cap) holding electrons at time t and their velocities v (not gamma v).
 * They are copied to the device, advanced nsteps particle steps in the
 * resident fields (each interior step with the null-collision MCC and
 * secondary birth; the last push ends at integer time without a collision
 * test), compacted, and copied back: positions in the axisymmetric frame at
 * azimuth 0 (x = r, y = 0), velocities in the matching local components.
 * *n_io is in/out; births may grow it up to cap rows (GASATT_E_CAPACITY if
 * more would be needed; the surplus is dropped). Pinned host memory gives
 * full copy bandwidth. */
int gasatt_sim_run_host(gasatt_sim *sim, double *pos, double *vel,
                        int64_t *n_io, int64_t cap, int nsteps);
/* cheap counter read (one small device->host copy) */
int gasatt_sim_counts(gasatt_sim *sim, int64_t *n_slots, int64_t *n_ionizations,
                      int64_t *n_lost);
/* device-side phase timing: with timing enabled the step graphs record CUDA
 * events around the field sub-cycle, the particle pass and (FP64 form) the
 * collision branch (commit + collision kernel, which runs beside the field
 * sub-cycle); last_timing gives their durations in the most recent step (ms).
 * The FP32 split form runs the collisions inside its particle pass and
 * reports mcc_ms = 0. */
int gasatt_sim_enable_timing(gasatt_sim *sim, int enable);
int gasatt_sim_last_timing(gasatt_sim *sim, float *fdtd_ms, float *pass_ms, float *mcc_ms);

/* ------------------------------------------------------------------ batches
 * Many independent gas cells (instances of uneven size, pressure, photon
 * energy) stepped together.  The reference's driver runs one cell at a time,
 * so this has no single counterpart there; it batches gasatt_sim_step.  All
 * instances belong to ctx and get the batch's sort period; each batch step
 * advances every instance by one step with one graph launch (their step
 * graphs side by side).  Each instance stays observable on its own
 * (gasatt_sim_read, gasatt_sim_diag, ...).  Destroy the batch before its
 * instances. */
typedef struct gasatt_batch gasatt_batch;
int gasatt_batch_create(gasatt_ctx *ctx, gasatt_sim *const *sims, int n, int sort_period,
                        gasatt_batch **batch);
int gasatt_batch_step(gasatt_batch *batch, int nsteps);
int gasatt_batch_destroy(gasatt_batch *batch);

#ifdef __cplusplus
}
#endif
#endif /* GASATT_H */
