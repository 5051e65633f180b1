/*
 * gasatt_mex.c - MATLAB MEX gateway of libgasatt: one MEX function
 *
 *     varargout = gasatt_mex(command, varargin)
 *
 * that stands in for the reference's parallel.gpu.CUDAKernel / feval calls
 * (electricmagneticfield6.m:77-111, electron_collision.m:4-8) and for its
 * MATLAB-side helpers, with the reference's argument lists:
 *
 *   gasatt_mex('init', device, seed)                       optional; default device 0, seed 0
 *   gasatt_mex('tables', t_el, t_sel, t_sel_1, t_del, t_sdel, t_ion, t_exc)
 *   [se, si, sx] = gasatt_mex('find_CS0', t_el, t_sel, t_ion, t_exc, E_PE)        find_CS0.m:1
 *   [xn, yn, zn, rn, phin] = gasatt_mex('free_motion', vx, vy, vz, x, y, z, dt)   free_motion.m:1
 *   [pos, vel, N_boundary] = gasatt_mex('REBOND', pos, r, phi, vel, Lp, PHIp)     REBOND.m:1
 *   d = gasatt_mex('particle_density', dr, dz, dphi, r, phi, z, cellnumxy,
 *                  sum_cell, VC, FN, ncell)                                      particle_density.m:1
 *   d = gasatt_mex('particle_density0', dr, dz, dphi, position, cellnumxy,
 *                  sum_cell, VC, FN, ncell)          position n x 3 (r, z, phi)   particle_density0.m:1
 *   [e_pos, e_vel, i1_pos, i1_vel, i2_pos, i2_vel, Er, Ez, Hphi, kin] =
 *       gasatt_mex('electricmagneticfield6', e_pos, e_vel, i1_pos, i1_vel, i2_pos,
 *                  i2_vel, Er, Ez, Hphi, delta, dt, Rp, Lp, PHIp, FN, cycle_time)  electricmagneticfield6.m:1
 *   [e_pos, e_vel, i1_pos, i1_vel] = gasatt_mex('electron_collision', e_pos, e_vel,
 *       i1_pos, i1_vel, t_el, t_sel_1, t_del, t_sdel, t_exc, electron_kinetic,
 *       sum_cell, cellnumxy, density, temperature, PHIp, phimax, dr, dz,
 *       sig_elastic, sig_ionization, sig_excitation, dt_transport)            electron_collision.m:1
 *   h = gasatt_mex('sim_create', cfg)        cfg: struct with gasatt_sim_config field names
 *   gasatt_mex('sim_load', h, r, z, ur, ut, uz, id)
 *   gasatt_mex('sim_birth_photo', h, n_photo, photon_keV, seed, sigma_r)
 *   gasatt_mex('sim_set_fields', h, Er, Ez, Hphi)     [Er, Ez, Hphi] = gasatt_mex('sim_get_fields', h)
 *   gasatt_mex('sim_set_gas_density', h, density)     density n_r x n_z, or [] for the uniform one
 *   gasatt_mex('sim_set_gas_temperature', h, T)       T n_r x n_z [K], or [] for the uniform one
 *   gasatt_mex('sim_load_ions', h, r, z, ur, ut, uz, id, charge)
 *   [r, z, ur, ut, uz, id, charge] = gasatt_mex('sim_read_ions', h)
 *   gasatt_mex('sim_step', h, nsteps)
 *   [r, z, ur, ut, uz, id] = gasatt_mex('sim_read', h)
 *   d = gasatt_mex('sim_diag', h)             struct with gasatt_diag field names
 *   gasatt_mex('sim_destroy', h)
 *
 * Particle and field arrays of the drop-ins are gpuArray (double) in and out;
 * tables, sizes and scalars are ordinary MATLAB values; the sim_* commands
 * take and return host arrays.  Outputs are allocated through
 * mxGPUCreateGPUArray, so MATLAB's gpuArray pool owns that memory, and the
 * density drop-in uses gasatt_particle_density_noalloc when the grid fits its
 * fixed array.  The drop-ins run with GASATT_FAITHFUL (the reference's
 * behaviour; see include/gasatt.h); 'electricmagneticfield6' takes positions
 * as (r, phi, z) columns like the reference (GASATT_POS_IN_CYL).
 *
 * Build (MATLAB R2018a or later, CUDA toolkit on the path):
 *     mexcuda -R2018a gasatt_mex.c -I<repo>/include -L<repo>/gas-atenuator_b200 -lgasatt
 */
#include <stdint.h>
#include <math.h>
#include <string.h>

#include <cuda_runtime.h>

#include "mex.h"
#include "gpu/mxGPUArray.h"
#include "gasatt.h"

static gasatt_ctx *g_ctx = NULL;
static gasatt_tables g_tab;
static double *g_tab_mem[7];

static void free_tables(void) {
  int k;
  for (k = 0; k < 7; ++k) {
    mxFree(g_tab_mem[k]);
    g_tab_mem[k] = NULL;
  }
  memset(&g_tab, 0, sizeof g_tab);
}

static void at_exit(void) {
  if (g_ctx) gasatt_destroy(g_ctx);
  g_ctx = NULL;
  free_tables();
}

static void fail(const char *what) {
  mexErrMsgIdAndTxt("gasatt:arg", "gasatt_mex: %s", what);
}

/* a library status: MATLAB error with the context's message */
static void check(int rc) {
  if (rc != GASATT_OK)
    mexErrMsgIdAndTxt("gasatt:call", "gasatt_mex: %s (status %d)",
                      g_ctx ? gasatt_last_error(g_ctx) : "no context", rc);
}

static void ensure_ctx(void) {
  if (!g_ctx) {
    check(gasatt_create(&g_ctx, 0, 0));
    mexAtExit(at_exit);
  }
}

static void nargs(int nrhs, int want, const char *usage) {
  if (nrhs != want) fail(usage);
}

static double scalar(const mxArray *a, const char *name) {
  if (!a || mxIsGPUArray(a) || !mxIsDouble(a) || mxGetNumberOfElements(a) != 1) fail(name);
  return mxGetScalar(a);
}

/* host double matrix (copied, so the library may keep no MATLAB pointer) */
static const double *host(const mxArray *a, const char *name) {
  if (!a || mxIsGPUArray(a) || !mxIsDouble(a) || mxIsComplex(a)) fail(name);
  return mxGetDoubles(a);
}

/* gpuArray in: a writable device copy (the drop-ins update in place) */
typedef struct {
  mxGPUArray *g;
  double *p;
  int64_t rows, cols;
} gpu_in;

static gpu_in gpu_copy(const mxArray *a, const char *name) {
  gpu_in r;
  const mwSize *dims;
  if (!mxIsGPUArray(a)) fail(name);
  r.g = mxGPUCopyFromMxArray(a);
  if (mxGPUGetClassID(r.g) != mxDOUBLE_CLASS || mxGPUGetComplexity(r.g) != mxREAL) {
    mxGPUDestroyGPUArray(r.g);
    fail(name);
  }
  dims = mxGPUGetDimensions(r.g);
  r.rows = (int64_t)dims[0];
  r.cols = mxGPUGetNumberOfDimensions(r.g) > 1 ? (int64_t)dims[1] : 1;
  mxFree((void *)dims);
  r.p = (double *)mxGPUGetData(r.g);
  return r;
}

static mxGPUArray *gpu_new(int64_t rows, int64_t cols, double **p) {
  mwSize d[2];
  mxGPUArray *g;
  d[0] = (mwSize)rows;
  d[1] = (mwSize)cols;
  g = mxGPUCreateGPUArray(2, d, mxDOUBLE_CLASS, mxREAL, MX_GPU_DO_NOT_INITIALIZE);
  *p = (double *)mxGPUGetData(g);
  return g;
}

static mxArray *gpu_out(mxGPUArray *g) {
  mxArray *a = mxGPUCreateMxArrayOnGPU(g);
  mxGPUDestroyGPUArray(g);
  return a;
}

/* the first n rows of an n_ld x c column-major device matrix as a new gpuArray */
static mxArray *gpu_rows(const double *src, int64_t ld, int64_t n, int64_t c) {
  double *dst;
  mxGPUArray *g = gpu_new(n, c, &dst);
  if (n > 0 && cudaMemcpy2D(dst, (size_t)n * 8, src, (size_t)ld * 8, (size_t)n * 8, (size_t)c,
                            cudaMemcpyDeviceToDevice) != cudaSuccess) {
    mxGPUDestroyGPUArray(g);
    fail("device copy failed");
  }
  return gpu_out(g);
}

static void need_tables(void) {
  if (!g_tab.t_el) fail("register the cross-section tables first: gasatt_mex('tables', ...)");
}

static void set_table(int k, const mxArray *a, const double **slot) {
  size_t n = mxGetNumberOfElements(a);
  mxFree(g_tab_mem[k]);
  g_tab_mem[k] = (double *)mxMalloc(n * sizeof(double) + 8);
  mexMakeMemoryPersistent(g_tab_mem[k]);
  memcpy(g_tab_mem[k], host(a, "tables must be double host matrices"), n * sizeof(double));
  *slot = g_tab_mem[k];
}

static void cmd_tables(int nrhs, const mxArray *prhs[]) {
  nargs(nrhs, 8, "tables(t_el, t_sel, t_sel_1, t_del, t_sdel, t_ion, t_exc)");
  set_table(0, prhs[1], &g_tab.t_el);   g_tab.n_el = (int)mxGetN(prhs[1]);
  set_table(1, prhs[2], &g_tab.t_sel);  g_tab.n_sel = (int)mxGetM(prhs[2]);
  set_table(2, prhs[3], &g_tab.t_sel_1); g_tab.n_sel1 = (int)mxGetM(prhs[3]);
  set_table(3, prhs[4], &g_tab.t_del);
  g_tab.del_rows = (int)mxGetM(prhs[4]); g_tab.del_cols = (int)mxGetN(prhs[4]);
  set_table(4, prhs[5], &g_tab.t_sdel);
  g_tab.sdel_rows = (int)mxGetM(prhs[5]); g_tab.sdel_cols = (int)mxGetN(prhs[5]);
  set_table(5, prhs[6], &g_tab.t_ion);  g_tab.n_ion = (int)mxGetM(prhs[6]);
  set_table(6, prhs[7], &g_tab.t_exc);  g_tab.n_exc = (int)mxGetM(prhs[7]);
}

static void cmd_find_cs0(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  gasatt_tables t;
  gpu_in E;
  double *se, *si, *sx;
  mxGPUArray *gs, *gi, *gx;
  nargs(nrhs, 6, "find_CS0(t_el, t_sel, t_ion, t_exc, E_PE)");
  need_tables();
  t = g_tab;                        /* the four tables of this call, the rest registered */
  t.t_el = host(prhs[1], "t_el");   t.n_el = (int)mxGetN(prhs[1]);
  t.t_sel = host(prhs[2], "t_sel"); t.n_sel = (int)mxGetM(prhs[2]);
  t.t_ion = host(prhs[3], "t_ion"); t.n_ion = (int)mxGetM(prhs[3]);
  t.t_exc = host(prhs[4], "t_exc"); t.n_exc = (int)mxGetM(prhs[4]);
  E = gpu_copy(prhs[5], "E_PE must be a double gpuArray");
  gs = gpu_new(E.rows, E.cols, &se);
  gi = gpu_new(E.rows, E.cols, &si);
  gx = gpu_new(E.rows, E.cols, &sx);
  check(gasatt_find_CS0(g_ctx, &t, E.p, E.rows * E.cols, se, si, sx, GASATT_FAITHFUL));
  mxGPUDestroyGPUArray(E.g);
  plhs[0] = gpu_out(gs);
  if (nlhs > 1) plhs[1] = gpu_out(gi); else mxGPUDestroyGPUArray(gi);
  if (nlhs > 2) plhs[2] = gpu_out(gx); else mxGPUDestroyGPUArray(gx);
}

static void cmd_free_motion(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  gpu_in a[6];
  double *o[5];
  mxGPUArray *g[5];
  int k;
  int64_t n;
  nargs(nrhs, 8, "free_motion(vx, vy, vz, x, y, z, dt)");
  for (k = 0; k < 6; ++k) a[k] = gpu_copy(prhs[1 + k], "vx..z must be double gpuArrays");
  n = a[0].rows * a[0].cols;
  for (k = 1; k < 6; ++k)
    if (a[k].rows * a[k].cols != n) fail("free_motion: arrays of different lengths");
  for (k = 0; k < 5; ++k) g[k] = gpu_new(a[0].rows, a[0].cols, &o[k]);
  check(gasatt_free_motion(g_ctx, a[0].p, a[1].p, a[2].p, a[3].p, a[4].p, a[5].p, n,
                           scalar(prhs[7], "dt"), o[0], o[1], o[2], o[3], o[4]));
  for (k = 0; k < 6; ++k) mxGPUDestroyGPUArray(a[k].g);
  for (k = 0; k < 5; ++k) {
    if (k < (nlhs > 0 ? nlhs : 1)) plhs[k] = gpu_out(g[k]);
    else mxGPUDestroyGPUArray(g[k]);
  }
}

static void cmd_rebond(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  gpu_in pos, r, phi, vel;
  int64_t nb = 0, n;
  nargs(nrhs, 7, "REBOND(particle_position, particle_r, particle_phi, particle_velocity, Lp, PHIp)");
  pos = gpu_copy(prhs[1], "particle_position must be a double gpuArray");
  r = gpu_copy(prhs[2], "particle_r must be a double gpuArray");
  phi = gpu_copy(prhs[3], "particle_phi must be a double gpuArray");
  vel = gpu_copy(prhs[4], "particle_velocity must be a double gpuArray");
  n = pos.rows;
  if ((n && pos.cols != 3) || vel.rows != n || (n && vel.cols != 3) || r.rows * r.cols != n ||
      phi.rows * phi.cols != n)
    fail("REBOND: positions and velocities n x 3, r and phi of length n");
  check(gasatt_rebond(g_ctx, pos.p, n, r.p, phi.p, vel.p, n, n, scalar(prhs[5], "Lp"),
                      scalar(prhs[6], "PHIp"), &nb));
  plhs[0] = mxGPUCreateMxArrayOnGPU(pos.g);
  if (nlhs > 1) plhs[1] = mxGPUCreateMxArrayOnGPU(vel.g);
  if (nlhs > 2) plhs[2] = mxCreateDoubleScalar((double)nb);
  mxGPUDestroyGPUArray(pos.g); mxGPUDestroyGPUArray(r.g);
  mxGPUDestroyGPUArray(phi.g); mxGPUDestroyGPUArray(vel.g);
}

/* particle_density's cell count: a positive integer, checked before MATLAB is
   asked for the output gpuArray */
static int64_t cell_count(const mxArray *a) {
  const double v = scalar(a, "ncell");
  if (!(v >= 1 && v <= 9.0e15) || v != floor(v)) fail("particle_density: ncell must be a positive integer");
  return (int64_t)v;
}

/* the density of particles at (r, phi, z) on the sector cells; the variant
   without device allocation leaves MATLAB's pool alone when the grid fits it */
static mxArray *density(const mxArray *dr, const mxArray *dz, const gpu_in *dphi,
                        const double *r, const double *phi, const double *z, int64_t n,
                        const mxArray *cellnumxy, const mxArray *sum_cell_a, const mxArray *VC_a,
                        const mxArray *FN, const mxArray *ncell_a) {
  gpu_in sum_cell = gpu_copy(sum_cell_a, "sum_cell must be a double gpuArray");
  gpu_in VC = gpu_copy(VC_a, "VC must be a double gpuArray");
  const int64_t ncell = cell_count(ncell_a);
  double *d;
  mxGPUArray *g = gpu_new(ncell, 1, &d);
  check((ncell <= GASATT_DENSITY_NOALLOC_MAX_CELLS ? gasatt_particle_density_noalloc
                                                    : gasatt_particle_density)(
      g_ctx, scalar(dr, "dr"), scalar(dz, "dz"), dphi->p, (int)(dphi->rows * dphi->cols), r, phi,
      z, n, (int)scalar(cellnumxy, "cellnumxy"), sum_cell.p, VC.p, ncell, scalar(FN, "FN"), d));
  mxGPUDestroyGPUArray(sum_cell.g); mxGPUDestroyGPUArray(VC.g);
  return gpu_out(g);
}

static void cmd_particle_density(mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  gpu_in dphi, r, phi, z;
  nargs(nrhs, 12, "particle_density(dr, dz, dphi, r, phi, z, cellnumxy, sum_cell, VC, FN, ncell)");
  cell_count(prhs[11]);
  dphi = gpu_copy(prhs[3], "dphi must be a double gpuArray");
  r = gpu_copy(prhs[4], "r must be a double gpuArray");
  phi = gpu_copy(prhs[5], "phi must be a double gpuArray");
  z = gpu_copy(prhs[6], "z must be a double gpuArray");
  plhs[0] = density(prhs[1], prhs[2], &dphi, r.p, phi.p, z.p, r.rows * r.cols, prhs[7], prhs[8],
                    prhs[9], prhs[10], prhs[11]);
  mxGPUDestroyGPUArray(dphi.g); mxGPUDestroyGPUArray(r.g); mxGPUDestroyGPUArray(phi.g);
  mxGPUDestroyGPUArray(z.g);
}

/* particle_density0.m: position columns (r, z, phi) */
static void cmd_particle_density0(mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  gpu_in dphi, pos;
  nargs(nrhs, 10, "particle_density0(dr, dz, dphi, position, cellnumxy, sum_cell, VC, FN, ncell)");
  cell_count(prhs[9]);
  dphi = gpu_copy(prhs[3], "dphi must be a double gpuArray");
  pos = gpu_copy(prhs[4], "position must be an n x 3 double gpuArray");
  if (pos.rows && pos.cols != 3) fail("particle_density0: position must be n x 3");
  plhs[0] = density(prhs[1], prhs[2], &dphi, pos.p, pos.p + 2 * pos.rows, pos.p + pos.rows,
                    pos.rows, prhs[5], prhs[6], prhs[7], prhs[8], prhs[9]);
  mxGPUDestroyGPUArray(dphi.g); mxGPUDestroyGPUArray(pos.g);
}

static void cmd_emf6(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  gpu_in s[9];
  int64_t n_e, n_i1, n_i2, out_e = 0, out_i1 = 0, out_i2 = 0;
  double *kin;
  mxGPUArray *gk;
  int k, n_r, n_z;
  nargs(nrhs, 17, "electricmagneticfield6(e_pos, e_vel, i1_pos, i1_vel, i2_pos, i2_vel, Er, Ez, "
                  "Hphi, delta, dt, Rp, Lp, PHIp, FN, cycle_time)");
  for (k = 0; k < 9; ++k) s[k] = gpu_copy(prhs[1 + k], "species and fields must be double gpuArrays");
  n_e = s[0].rows; n_i1 = s[2].rows; n_i2 = s[4].rows;
  if (s[1].rows != n_e || s[3].rows != n_i1 || s[5].rows != n_i2 ||
      (n_e && (s[0].cols != 3 || s[1].cols != 3)) || (n_i1 && (s[2].cols != 3 || s[3].cols != 3)) ||
      (n_i2 && (s[4].cols != 3 || s[5].cols != 3)))
    fail("electricmagneticfield6: species must be n x 3");
  n_r = (int)s[8].rows; n_z = (int)s[8].cols;
  gk = gpu_new(n_e, 1, &kin);
  check(gasatt_electricmagneticfield6(
      g_ctx, s[0].p, s[1].p, n_e, s[2].p, s[3].p, n_i1, s[4].p, s[5].p, n_i2, s[6].p, s[7].p,
      s[8].p, n_r, n_z, scalar(prhs[10], "delta"), scalar(prhs[11], "dt"), scalar(prhs[12], "Rp"),
      scalar(prhs[13], "Lp"), scalar(prhs[14], "PHIp"), scalar(prhs[15], "FN"),
      (int)scalar(prhs[16], "cycle_time"), kin, &out_e, &out_i1, &out_i2,
      GASATT_FAITHFUL | GASATT_POS_IN_CYL));
  {
    const int64_t ld[6] = {n_e, n_e, n_i1, n_i1, n_i2, n_i2};
    const int64_t nout[6] = {out_e, out_e, out_i1, out_i1, out_i2, out_i2};
    for (k = 0; k < 6; ++k)
      if (k < nlhs || k == 0) plhs[k] = gpu_rows(s[k].p, ld[k], nout[k], 3);
  }
  for (k = 6; k < 9; ++k) {
    if (k < nlhs) plhs[k] = mxGPUCreateMxArrayOnGPU(s[k].g);
  }
  if (nlhs > 9) plhs[9] = gpu_rows(kin, n_e, out_e, 1);
  mxGPUDestroyGPUArray(gk);
  for (k = 0; k < 9; ++k) mxGPUDestroyGPUArray(s[k].g);
}

static void cmd_collision(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  gpu_in ep, ev, ip, iv, kin, dens, temp, se, si, sx;
  gasatt_tables t;
  double *e_pos, *e_vel, *i_pos, *i_vel;
  mxGPUArray *g[4];
  int64_t n_e, n_i1, out_e = 0, out_i1 = 0;
  int rmax, k;
  nargs(nrhs, 23, "electron_collision(e_pos, e_vel, i1_pos, i1_vel, t_el, t_sel_1, t_del, t_sdel, "
                  "t_exc, electron_kinetic, sum_cell, cellnumxy, density, temperature, PHIp, "
                  "phimax, dr, dz, sig_elastic, sig_ionization, sig_excitation, dt_transport)");
  need_tables();
  t = g_tab;
  t.t_el = host(prhs[5], "t_el");       t.n_el = (int)mxGetN(prhs[5]);
  t.t_sel_1 = host(prhs[6], "t_sel_1"); t.n_sel1 = (int)mxGetM(prhs[6]);
  t.t_del = host(prhs[7], "t_del");
  t.del_rows = (int)mxGetM(prhs[7]);    t.del_cols = (int)mxGetN(prhs[7]);
  t.t_sdel = host(prhs[8], "t_sdel");
  t.sdel_rows = (int)mxGetM(prhs[8]);   t.sdel_cols = (int)mxGetN(prhs[8]);
  t.t_exc = host(prhs[9], "t_exc");     t.n_exc = (int)mxGetM(prhs[9]);
  ep = gpu_copy(prhs[1], "e_pos"); ev = gpu_copy(prhs[2], "e_vel");
  ip = gpu_copy(prhs[3], "i1_pos"); iv = gpu_copy(prhs[4], "i1_vel");
  kin = gpu_copy(prhs[10], "electron_kinetic");
  dens = gpu_copy(prhs[13], "density"); temp = gpu_copy(prhs[14], "temperature");
  se = gpu_copy(prhs[19], "sig_elastic"); si = gpu_copy(prhs[20], "sig_ionization");
  sx = gpu_copy(prhs[21], "sig_excitation");
  n_e = ep.rows; n_i1 = ip.rows;
  if (ev.rows != n_e || iv.rows != n_i1) fail("electron_collision: positions and velocities differ");
  /* room for one secondary electron and one ion per electron */
  g[0] = gpu_new(2 * n_e, 3, &e_pos); g[1] = gpu_new(2 * n_e, 3, &e_vel);
  g[2] = gpu_new(n_i1 + n_e, 3, &i_pos); g[3] = gpu_new(n_i1 + n_e, 3, &i_vel);
  for (k = 0; k < 3; ++k) {
    if (n_e) {
      cudaMemcpy(e_pos + k * 2 * n_e, ep.p + k * n_e, (size_t)n_e * 8, cudaMemcpyDeviceToDevice);
      cudaMemcpy(e_vel + k * 2 * n_e, ev.p + k * n_e, (size_t)n_e * 8, cudaMemcpyDeviceToDevice);
    }
    if (n_i1) {
      cudaMemcpy(i_pos + k * (n_i1 + n_e), ip.p + k * n_i1, (size_t)n_i1 * 8, cudaMemcpyDeviceToDevice);
      cudaMemcpy(i_vel + k * (n_i1 + n_e), iv.p + k * n_i1, (size_t)n_i1 * 8, cudaMemcpyDeviceToDevice);
    }
  }
  rmax = (int)mxGetNumberOfElements(prhs[11]);
  check(gasatt_electron_collision(
      g_ctx, e_pos, e_vel, n_e, 2 * n_e, i_pos, i_vel, n_i1, n_i1 + n_e, &t, kin.p,
      host(prhs[11], "sum_cell"), rmax, (int)scalar(prhs[12], "cellnumxy"), dens.p, temp.p,
      dens.rows * dens.cols, scalar(prhs[15], "PHIp"), host(prhs[16], "phimax"),
      scalar(prhs[17], "dr"), scalar(prhs[18], "dz"), se.p, si.p, sx.p,
      scalar(prhs[22], "dt_transport"), NULL, &out_e, &out_i1, GASATT_FAITHFUL));
  plhs[0] = gpu_rows(e_pos, 2 * n_e, out_e, 3);
  if (nlhs > 1) plhs[1] = gpu_rows(e_vel, 2 * n_e, out_e, 3);
  if (nlhs > 2) plhs[2] = gpu_rows(i_pos, n_i1 + n_e, out_i1, 3);
  if (nlhs > 3) plhs[3] = gpu_rows(i_vel, n_i1 + n_e, out_i1, 3);
  for (k = 0; k < 4; ++k) mxGPUDestroyGPUArray(g[k]);
  mxGPUDestroyGPUArray(ep.g); mxGPUDestroyGPUArray(ev.g); mxGPUDestroyGPUArray(ip.g);
  mxGPUDestroyGPUArray(iv.g); mxGPUDestroyGPUArray(kin.g); mxGPUDestroyGPUArray(dens.g);
  mxGPUDestroyGPUArray(temp.g); mxGPUDestroyGPUArray(se.g); mxGPUDestroyGPUArray(si.g);
  mxGPUDestroyGPUArray(sx.g);
}

/* ------------------------------------------------------------ resident sim */
static gasatt_sim *sim_of(const mxArray *a) {
  if (!a || !mxIsUint64(a) || mxGetNumberOfElements(a) != 1) fail("not a simulation handle");
  return (gasatt_sim *)(uintptr_t)(*(const uint64_t *)mxGetData(a));
}

/* fields of gasatt_sim_config settable from a MATLAB struct, by C type */
#define CFG_DOUBLES(X) X(dr) X(dz) X(dt) X(PHIp) X(FN) X(gas_density) X(gas_temperature) \
  X(q_e) X(m_e) X(c) X(eps0) X(mu0) X(kb) X(m_ion) X(table_emin_ev) X(table_emax_ev)
#define CFG_INTS(X) X(n_r) X(n_z) X(fdtd_ratio) X(precision) X(sort_period) X(secondaries) \
  X(table_n) X(ion_subcycle)
#define CFG_INT64S(X) X(capacity) X(ion_capacity)

static void cmd_sim_create(mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  gasatt_sim_config cfg;
  gasatt_sim *s = NULL;
  const mxArray *f;
  nargs(nrhs, 2, "sim_create(cfg)");
  if (!mxIsStruct(prhs[1])) fail("sim_create: cfg must be a struct");
  need_tables();
  check(gasatt_sim_default_config(&cfg));
#define SET_D(name) if ((f = mxGetField(prhs[1], 0, #name)) != NULL) cfg.name = scalar(f, #name);
#define SET_I(name) if ((f = mxGetField(prhs[1], 0, #name)) != NULL) cfg.name = (int)scalar(f, #name);
#define SET_L(name) if ((f = mxGetField(prhs[1], 0, #name)) != NULL) cfg.name = (int64_t)scalar(f, #name);
  CFG_DOUBLES(SET_D)
  CFG_INTS(SET_I)
  CFG_INT64S(SET_L)
#undef SET_D
#undef SET_I
#undef SET_L
  if ((f = mxGetField(prhs[1], 0, "seed")) != NULL) cfg.seed = (uint64_t)scalar(f, "seed");
  if ((f = mxGetField(prhs[1], 0, "flags")) != NULL) cfg.flags = (unsigned)scalar(f, "flags");
  check(gasatt_sim_create(g_ctx, &cfg, &g_tab, &s));
  plhs[0] = mxCreateNumericMatrix(1, 1, mxUINT64_CLASS, mxREAL);
  *(uint64_t *)mxGetData(plhs[0]) = (uint64_t)(uintptr_t)s;
}

static void cmd_sim_load(int nrhs, const mxArray *prhs[]) {
  const double *a[5];
  size_t n;
  int k;
  nargs(nrhs, 8, "sim_load(h, r, z, ur, ut, uz, id)");
  n = mxGetNumberOfElements(prhs[2]);
  for (k = 0; k < 5; ++k) {
    a[k] = host(prhs[2 + k], "r..uz must be double host arrays");
    if (mxGetNumberOfElements(prhs[2 + k]) != n) fail("sim_load: arrays of different lengths");
  }
  if (!mxIsUint64(prhs[7]) || mxGetNumberOfElements(prhs[7]) != n) fail("sim_load: id must be uint64");
  check(gasatt_sim_load(sim_of(prhs[1]), a[0], a[1], a[2], a[3], a[4],
                        (const uint64_t *)mxGetData(prhs[7]), (int64_t)n, 0));
}

static void cmd_sim_fields(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[], int set) {
  gasatt_sim *s;
  gasatt_sim_config cfg;
  size_t nr, nz;
  int k;
  if (set) nargs(nrhs, 5, "sim_set_fields(h, Er, Ez, Hphi)");
  else nargs(nrhs, 2, "sim_get_fields(h)");
  s = sim_of(prhs[1]);
  check(gasatt_sim_get_config(s, &cfg));
  nr = (size_t)cfg.n_r; nz = (size_t)cfg.n_z;
  if (set) {
    const double *f[3];
    if (mxGetM(prhs[2]) != nr || mxGetN(prhs[2]) != nz + 1 || mxGetM(prhs[3]) != nr + 1 ||
        mxGetN(prhs[3]) != nz || mxGetM(prhs[4]) != nr || mxGetN(prhs[4]) != nz)
      fail("sim_set_fields: Er n_r x (n_z+1), Ez (n_r+1) x n_z, Hphi n_r x n_z");
    for (k = 0; k < 3; ++k) f[k] = host(prhs[2 + k], "fields must be double host matrices");
    check(gasatt_sim_set_fields(s, f[0], f[1], f[2], 0));
  } else {
    mxArray *o[3];
    o[0] = mxCreateDoubleMatrix(nr, nz + 1, mxREAL);
    o[1] = mxCreateDoubleMatrix(nr + 1, nz, mxREAL);
    o[2] = mxCreateDoubleMatrix(nr, nz, mxREAL);
    check(gasatt_sim_get_fields(s, mxGetDoubles(o[0]), mxGetDoubles(o[1]), mxGetDoubles(o[2]), 0));
    for (k = 0; k < 3; ++k) {
      if (k < (nlhs > 0 ? nlhs : 1)) plhs[k] = o[k];
      else mxDestroyArray(o[k]);
    }
  }
}

/* a per-cell gas map (density or temperature), n_r x n_z; [] = uniform */
static void cmd_sim_gas(int nrhs, const mxArray *prhs[], int temperature) {
  gasatt_sim *s;
  gasatt_sim_config cfg;
  const double *m = NULL;
  nargs(nrhs, 3, temperature ? "sim_set_gas_temperature(h, T)" : "sim_set_gas_density(h, density)");
  s = sim_of(prhs[1]);
  check(gasatt_sim_get_config(s, &cfg));
  if (mxGetNumberOfElements(prhs[2]) != 0) {
    if (mxGetM(prhs[2]) != (size_t)cfg.n_r || mxGetN(prhs[2]) != (size_t)cfg.n_z)
      fail("gas map must be n_r x n_z");
    m = host(prhs[2], "gas map must be a double host matrix");
  }
  check(temperature ? gasatt_sim_set_gas_temperature(s, m, 0) : gasatt_sim_set_gas_density(s, m, 0));
}

static void cmd_sim_load_ions(int nrhs, const mxArray *prhs[]) {
  const double *a[5];
  const int8_t *q = NULL;
  int8_t *qbuf = NULL;
  size_t n, k;
  nargs(nrhs, 9, "sim_load_ions(h, r, z, ur, ut, uz, id, charge)");
  n = mxGetNumberOfElements(prhs[2]);
  for (k = 0; k < 5; ++k) {
    a[k] = host(prhs[2 + k], "r..uz must be double host arrays");
    if (mxGetNumberOfElements(prhs[2 + k]) != n) fail("sim_load_ions: arrays of different lengths");
  }
  if (!mxIsUint64(prhs[7]) || mxGetNumberOfElements(prhs[7]) != n) fail("sim_load_ions: id must be uint64");
  if (mxGetNumberOfElements(prhs[8]) > 0) {                /* charge numbers as doubles; [] = all 1 */
    const double *c = host(prhs[8], "charge must be a double host array");
    if (mxGetNumberOfElements(prhs[8]) != n) fail("sim_load_ions: charge of another length");
    qbuf = (int8_t *)mxMalloc(n ? n : 1);
    for (k = 0; k < n; ++k) qbuf[k] = (int8_t)c[k];
    q = qbuf;
  }
  {
    const int rc = gasatt_sim_load_ions(sim_of(prhs[1]), a[0], a[1], a[2], a[3], a[4],
                                        (const uint64_t *)mxGetData(prhs[7]), q, (int64_t)n, 0);
    mxFree(qbuf);
    check(rc);
  }
}

static void cmd_sim_read_ions(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  gasatt_sim *s;
  int64_t n = 0, k;
  double *p[5];
  int8_t *q;
  mxArray *o[7];
  nargs(nrhs, 2, "sim_read_ions(h)");
  s = sim_of(prhs[1]);
  gasatt_sim_read_ions(s, NULL, NULL, NULL, NULL, NULL, NULL, NULL, 0, &n, 0);   /* count only */
  for (k = 0; k < 5; ++k) {
    o[k] = mxCreateDoubleMatrix((mwSize)n, 1, mxREAL);
    p[k] = mxGetDoubles(o[k]);
  }
  o[5] = mxCreateNumericMatrix((mwSize)n, 1, mxUINT64_CLASS, mxREAL);
  o[6] = mxCreateDoubleMatrix((mwSize)n, 1, mxREAL);
  q = (int8_t *)mxMalloc(n ? (size_t)n : 1);
  {
    const int rc = gasatt_sim_read_ions(s, p[0], p[1], p[2], p[3], p[4],
                                        (uint64_t *)mxGetData(o[5]), q, n, &n, 0);
    for (k = 0; k < n; ++k) mxGetDoubles(o[6])[k] = (double)q[k];
    mxFree(q);
    check(rc);
  }
  for (k = 0; k < 7; ++k) {
    if (k < (nlhs > 0 ? nlhs : 1)) plhs[k] = o[k];
    else mxDestroyArray(o[k]);
  }
}

static void cmd_sim_read(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  gasatt_sim *s;
  int64_t n = 0;
  double *p[5];
  mxArray *o[6];
  int k;
  nargs(nrhs, 2, "sim_read(h)");
  s = sim_of(prhs[1]);
  gasatt_sim_read(s, NULL, NULL, NULL, NULL, NULL, NULL, 0, &n, 0);   /* count only */
  for (k = 0; k < 5; ++k) {
    o[k] = mxCreateDoubleMatrix((mwSize)n, 1, mxREAL);
    p[k] = mxGetDoubles(o[k]);
  }
  o[5] = mxCreateNumericMatrix((mwSize)n, 1, mxUINT64_CLASS, mxREAL);
  check(gasatt_sim_read(s, p[0], p[1], p[2], p[3], p[4], (uint64_t *)mxGetData(o[5]), n, &n, 0));
  for (k = 0; k < 6; ++k) {
    if (k < (nlhs > 0 ? nlhs : 1)) plhs[k] = o[k];
    else mxDestroyArray(o[k]);
  }
}

static void cmd_sim_diag(mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  static const char *names[] = {"n_alive", "n_total", "n_ionizations", "n_elastic",
                                "n_excitation", "n_null", "n_lost_wall", "n_ions",
                                "kinetic_ev", "field_energy_j", "steps", "status_flags",
                                "n_ion_lost_wall", "ion_kinetic_ev", "net_charge_c",
                                "collision_loss_ev", "wall_loss_ev"};
  gasatt_diag d;
  double w[17];
  int k;
  nargs(nrhs, 2, "sim_diag(h)");
  check(gasatt_sim_diag(sim_of(prhs[1]), &d));
  w[0] = (double)d.n_alive; w[1] = (double)d.n_total; w[2] = (double)d.n_ionizations;
  w[3] = (double)d.n_elastic; w[4] = (double)d.n_excitation; w[5] = (double)d.n_null;
  w[6] = (double)d.n_lost_wall; w[7] = (double)d.n_ions; w[8] = d.kinetic_ev;
  w[9] = d.field_energy_j; w[10] = (double)d.steps; w[11] = (double)d.status_flags;
  w[12] = (double)d.n_ion_lost_wall; w[13] = d.ion_kinetic_ev; w[14] = d.net_charge_c;
  w[15] = d.collision_loss_ev; w[16] = d.wall_loss_ev;
  plhs[0] = mxCreateStructMatrix(1, 1, 17, names);
  for (k = 0; k < 17; ++k) mxSetField(plhs[0], 0, names[k], mxCreateDoubleScalar(w[k]));
}

static const char *const k_commands[] = {
    "init", "tables", "find_CS0", "free_motion", "REBOND", "particle_density", "particle_density0",
    "electricmagneticfield6",
    "electron_collision", "sim_create", "sim_load", "sim_step", "sim_read", "sim_diag",
    "sim_destroy", "sim_birth_photo", "sim_set_fields", "sim_get_fields", "sim_set_gas_density",
    "sim_set_gas_temperature",
    "sim_load_ions", "sim_read_ions"};

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  char cmd[64];
  size_t k;
  int known = 0;
  if (nrhs < 1 || !mxIsChar(prhs[0]) || mxGetString(prhs[0], cmd, sizeof cmd))
    fail("first argument: command name");
  for (k = 0; k < sizeof k_commands / sizeof k_commands[0]; ++k)
    known = known || !strcmp(cmd, k_commands[k]);
  if (!known) fail("unknown command");
  if (!strcmp(cmd, "tables")) { cmd_tables(nrhs, prhs); return; }
  mxInitGPU();
  if (!strcmp(cmd, "init")) {
    int dev = nrhs > 1 ? (int)scalar(prhs[1], "device") : 0;
    uint64_t seed = nrhs > 2 ? (uint64_t)scalar(prhs[2], "seed") : 0;
    if (g_ctx) gasatt_destroy(g_ctx);
    g_ctx = NULL;
    check(gasatt_create(&g_ctx, dev, seed));
    mexAtExit(at_exit);
    return;
  }
  ensure_ctx();
  if (!strcmp(cmd, "find_CS0")) cmd_find_cs0(nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "free_motion")) cmd_free_motion(nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "REBOND")) cmd_rebond(nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "particle_density")) cmd_particle_density(plhs, nrhs, prhs);
  else if (!strcmp(cmd, "particle_density0")) cmd_particle_density0(plhs, nrhs, prhs);
  else if (!strcmp(cmd, "electricmagneticfield6")) cmd_emf6(nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "electron_collision")) cmd_collision(nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "sim_create")) cmd_sim_create(plhs, nrhs, prhs);
  else if (!strcmp(cmd, "sim_load")) cmd_sim_load(nrhs, prhs);
  else if (!strcmp(cmd, "sim_step")) {
    nargs(nrhs, 3, "sim_step(h, nsteps)");
    check(gasatt_sim_step(sim_of(prhs[1]), (int)scalar(prhs[2], "nsteps")));
  } else if (!strcmp(cmd, "sim_read")) cmd_sim_read(nlhs, plhs, nrhs, prhs);
  else if (!strcmp(cmd, "sim_diag")) cmd_sim_diag(plhs, nrhs, prhs);
  else if (!strcmp(cmd, "sim_birth_photo")) {
    nargs(nrhs, 6, "sim_birth_photo(h, n_photo, photon_keV, seed, sigma_r)");
    check(gasatt_sim_birth_photo(sim_of(prhs[1]), (int64_t)scalar(prhs[2], "n_photo"),
                                 scalar(prhs[3], "photon_keV"), scalar(prhs[5], "sigma_r"),
                                 (uint64_t)scalar(prhs[4], "seed"), 0));
  } else if (!strcmp(cmd, "sim_set_fields")) cmd_sim_fields(nlhs, plhs, nrhs, prhs, 1);
  else if (!strcmp(cmd, "sim_get_fields")) cmd_sim_fields(nlhs, plhs, nrhs, prhs, 0);
  else if (!strcmp(cmd, "sim_set_gas_density")) cmd_sim_gas(nrhs, prhs, 0);
  else if (!strcmp(cmd, "sim_set_gas_temperature")) cmd_sim_gas(nrhs, prhs, 1);
  else if (!strcmp(cmd, "sim_load_ions")) cmd_sim_load_ions(nrhs, prhs);
  else if (!strcmp(cmd, "sim_read_ions")) cmd_sim_read_ions(nlhs, plhs, nrhs, prhs);
  else {
    nargs(nrhs, 2, "sim_destroy(h)");
    check(gasatt_sim_destroy(sim_of(prhs[1])));
  }
}
