/*
 * gasatt_oracle.c - CPU FP64 oracle of the PIC-MCC electron step.
 *
 * TEST INFRASTRUCTURE ONLY (checker for tests/, the smoke check and bench.py's
 * CPU baseline).  The product library does not link or call this file.
 *
 * Plain C restatement of the reference:
 *   EM2.cu, EM7.cu, EM3_1.cu, EM3.cu, EM4.cu           (push / deposit / FDTD kernels)
 *   electron_transport.cu                              (MCC kernel)
 *   electricmagneticfield6.m, electron_collision.m     (their MATLAB orchestration)
 *   find_CS0.m, free_motion.m, particle_density.m      (MATLAB drop-ins)
 *   get_ElasticSc_sub1.m, get_ImpIonized.m, get_ImpExc2.m, rotate.m (CPU-path MCC pieces)
 * MATLAB built-ins are restated from their documented definitions: interp1
 * (linear, NaN outside the knots), cumtrapz (trapezoid rule), round (half away
 * from zero).
 */
#include "gasatt_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 1;
void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int  orc_get_threads(void) { return g_threads; }

/* ===================================================================== RNG */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies with the
 * published multipliers and Weyl key increments. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int i = 0; i < 10; ++i) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c1 = (uint32_t)p1;
    c3 = (uint32_t)p0;
    c0 = n0;
    c2 = n2;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* (2b+1) 2^-53 with b the top 52 bits: exact, in (0, 1) */
double orc_u01(uint32_t hi, uint32_t lo) {
  uint64_t b = ((((uint64_t)hi) << 32) | lo) >> 12;
  return (double)b * 0x1.0p-52 + 0x1.0p-53;
}

/* splitmix64 finaliser over (parent id, step): identity of a secondary */
uint64_t orc_child_id(uint64_t parent, int64_t step) {
  uint64_t z = parent + 0x9E3779B97F4A7C15ull * (uint64_t)(step + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static void draw_block(uint64_t seed, uint64_t id, int64_t step, uint32_t blk, double *ua, double *ub) {
  uint32_t ctr[4] = {(uint32_t)id, (uint32_t)(id >> 32), (uint32_t)step, blk};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  orc_philox4x32_10(ctr, key, o);
  *ua = orc_u01(o[0], o[1]);
  *ub = orc_u01(o[2], o[3]);
}

/* ========================================================== MATLAB interp1 */
/* interp1(x, y, xq) 'linear': NaN outside [x(1), x(end)]. */
double orc_interp1(const double *x, int sx, const double *y, int sy, int n, double xq) {
  if (!(xq >= x[0] && xq <= x[(int64_t)(n - 1) * sx])) return NAN;
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (x[(int64_t)mid * sx] <= xq) lo = mid; else hi = mid;
  }
  double x0 = x[(int64_t)lo * sx], x1 = x[(int64_t)hi * sx];
  double y0 = y[(int64_t)lo * sy], y1 = y[(int64_t)hi * sy];
  return y0 + (xq - x0) * (y1 - y0) / (x1 - x0);
}

/* log-log extrapolation beyond the last knot (corrected policy) */
static double loglog_tail(const double *x, int sx, const double *y, int sy, int n, double xq) {
  double x0 = x[(int64_t)(n - 2) * sx], x1 = x[(int64_t)(n - 1) * sx];
  double y0 = y[(int64_t)(n - 2) * sy], y1 = y[(int64_t)(n - 1) * sy];
  double s = log(y1 / y0) / log(x1 / x0);
  return y1 * pow(xq / x1, s);
}

/* ================================================================ find_CS0 */
/* find_CS0.m:1-61.  Corrected policy (flag GASATT_Q_XS_NAN clear):
 *   sigma_el below the first low-energy knot (1 eV) holds the knot value,
 *   sigma_el and sigma_ion above 20 keV follow a log-log tail,
 *   sigma_ion is 0 at or below its first knot (15.6 eV),
 *   each excitation term is 0 at or below its threshold k_j. */
static void cs0_one(const gasatt_tables *t, double E, double *se, double *si, double *sx,
                    unsigned flags) {
  const int faithful = (flags & GASATT_Q_XS_NAN) != 0;
  const double *t_el = t->t_el; const int n_el = t->n_el;
  const double *t_sel = t->t_sel; const int n_sel = t->n_sel;
  const double *t_ion = t->t_ion; const int n_ion = t->n_ion;
  const double *t_exc = t->t_exc; const int n_exc = t->n_exc;
  double sel = 0.0;
  if (E >= 0.05) {                                    /* find_CS0.m:102-107 */
    sel = orc_interp1(&t_el[0], 2, &t_el[1], 2, n_el, E);
    if (!faithful && E > t_el[2 * (n_el - 1)])
      sel = loglog_tail(&t_el[0], 2, &t_el[1], 2, n_el, E);
    sel = sel * GASATT_A0SQ * 2;
  } else if (E < 0.05) {                              /* find_CS0.m:108-111 */
    double Ev = E * 1000;
    if (!faithful && Ev < t_sel[0]) Ev = t_sel[0];
    sel = orc_interp1(&t_sel[0], 1, &t_sel[n_sel], 1, n_sel, Ev) * 1e-20;
  }
  *se = sel;
  double T = E * 1000;                                /* find_CS0.m:116-119 */
  double sion;
  if (!faithful && T <= t_ion[0]) sion = 0.0;
  else if (!faithful && T > t_ion[n_ion - 1])
    sion = loglog_tail(&t_ion[0], 1, &t_ion[n_ion], 1, n_ion, T) * 1e-20;
  else sion = orc_interp1(&t_ion[0], 1, &t_ion[n_ion], 1, n_ion, T) * 1e-20;
  *si = sion;
  double sexc = 0.0;                                  /* find_CS0.m:123-142 */
  for (int i = 0; i < n_exc; ++i) {
    double k = t_exc[i], A = t_exc[n_exc + i], om = t_exc[2 * n_exc + i];
    double nu = t_exc[3 * n_exc + i], ga = t_exc[4 * n_exc + i];
    if (!faithful && !(T > k)) continue;
    double a = GASATT_CS_Q0 * A / (k * k);
    double b = pow(k / T, om);
    double c = pow(1 - pow(k / T, ga), nu);
    sexc = sexc + a * b * c;
  }
  *sx = sexc * 1e-4;
}

void orc_find_cs0(const gasatt_tables *t, const double *E, int64_t n, double *s_el,
                  double *s_ion, double *s_exc, unsigned flags) {
  for (int64_t i = 0; i < n; ++i) cs0_one(t, E[i], &s_el[i], &s_ion[i], &s_exc[i], flags);
}

/* electron_collision.m:12-33: combined elastic TCS (yInterp, a0^2 per atom),
 * log energies of the DCS columns (xInterp) and log DCS (V_interp, 181 x ne). */
int orc_elastic_tables(const gasatt_tables *t, double *xInterp, double *yInterp, double *V_interp) {
  const int m1 = t->n_sel1 - 1;
  const int ne = m1 + t->n_el;
  if (t->del_rows != 182 || t->sdel_rows != 182) return -1;
  if ((t->sdel_cols - 1) + (t->del_cols - 1) != ne) return -2;
  for (int i = 0; i < m1; ++i)                          /* :15-17 */
    yInterp[i] = t->t_sel_1[t->n_sel1 + i] * 1e-20 / GASATT_A0SQ / 2;
  for (int i = 0; i < t->n_el; ++i) yInterp[m1 + i] = t->t_el[2 * i + 1];   /* :19-20,33 */
  /* t_del = [t_sdel, t_del(:,2:end)]; E = t_del(1,2:end); DCS = t_del(2:end,2:end) */
  int col = 0;
  for (int c = 1; c < t->sdel_cols; ++c, ++col) {
    xInterp[col] = log(t->t_sdel[(int64_t)c * 182]);
    for (int k = 0; k < 181; ++k)
      V_interp[(int64_t)col * 181 + k] = log(t->t_sdel[(int64_t)c * 182 + 1 + k]);
  }
  for (int c = 1; c < t->del_cols; ++c, ++col) {
    xInterp[col] = log(t->t_del[(int64_t)c * 182]);
    for (int k = 0; k < 181; ++k)
      V_interp[(int64_t)col * 181 + k] = log(t->t_del[(int64_t)c * 182 + 1 + k]);
  }
  return ne;
}

/* ============================================================ EM2 / EM4 drift */
/* EM2.cu:26-57 (and EM4.cu:146-177): half drift, (r, phi), wall delete,
 * wedge wrap rotating the velocity-like vector w, specular z. */
static void halfdrift_cart(double *x, double *y, double *z, double *wx, double *wy, double *wz,
                           double vx, double vy, double vz, double *r_o, double *phi_o,
                           int *del, double Rp, double Lp, double PHIp, double dt,
                           unsigned flags) {
  double X = *x + 0.5 * vx * dt;
  double Y = *y + 0.5 * vy * dt;
  double Z = *z + 0.5 * vz * dt;
  double r = sqrt(X * X + Y * Y);
  double phi = (flags & GASATT_Q_ATAN_PHI) ? atan(Y / X) : atan2(Y, X);
  if (r > Rp) *del = 1;
  const int wrap = (flags & GASATT_Q_ATAN_PHI) || PHIp < 2 * GASATT_PI - 1e-12;
  if (wrap) {
    double cp = cos(PHIp), sp = sin(PHIp), w1;
    while (phi < 0) {
      phi = phi + PHIp;
      w1 = *wx * cp - *wy * sp;
      *wy = *wx * sp + *wy * cp;
      *wx = w1;
    }
    while (phi > PHIp) {
      phi = phi - PHIp;
      w1 = *wx * cp + *wy * sp;
      *wy = -*wx * sp + *wy * cp;
      *wx = w1;
    }
  }
  X = r * cos(phi);
  Y = r * sin(phi);
  if (Z > Lp) { Z = 2 * Lp - Z; *wz = -*wz; }
  if (Z < 0) { Z = -Z; *wz = -*wz; }
  *x = X; *y = Y; *z = Z;
  *r_o = r; *phi_o = phi;
}

void orc_em2(double *x, double *y, double *z, double *vx, double *vy, double *vz,
             double *r, double *phi, double *vr, int *del, int64_t n,
             double Rp, double Lp, double PHIp, double dt, unsigned flags) {
  for (int64_t i = 0; i < n; ++i) {
    if (del[i] == 1) continue;                           /* EM2.cu:23 */
    halfdrift_cart(&x[i], &y[i], &z[i], &vx[i], &vy[i], &vz[i], vx[i], vy[i], vz[i],
                   &r[i], &phi[i], &del[i], Rp, Lp, PHIp, dt, flags);
    vr[i] = vx[i] * cos(phi[i]) + vy[i] * sin(phi[i]);   /* EM2.cu:57 */
  }
}

/* =============================================================== EM7 deposit */
/* EM7.cu:56-176: node indices a[4] and bilinear weights b[4] on the
 * cell-centred grid with one-sided edge cases; shell volumes V1 (column ar)
 * and V2 (column ar+1). */
static void em7_weights(double r0, double z0, int nr, int nz, double dr, double dz,
                        int64_t a[4], double b[4], int *ar_o) {
  int ar = (int)floor(r0 / dr - 0.5);
  int az = (int)floor(z0 / dz - 0.5);
  *ar_o = ar;
  a[0] = a[1] = a[2] = a[3] = 0;
  b[0] = b[1] = b[2] = b[3] = 0;
  if (ar < 0) {
    if (az < 0) { a[3] = (ar + 1) + (int64_t)(az + 1) * nr; b[3] = 1; }
    else if (az >= nz - 1) { a[1] = (ar + 1) + (int64_t)az * nr; b[1] = 1; }
    else {
      a[1] = (ar + 1) + (int64_t)az * nr; a[3] = (ar + 1) + (int64_t)(az + 1) * nr;
      b[1] = ((az + 1.5) * dz - z0) / (dz);
      b[3] = (z0 - (az + 0.5) * dz) / (dz);
    }
  } else if (ar >= nr - 1) {
    if (az < 0) { a[2] = ar + (int64_t)(az + 1) * nr; b[2] = 1; }
    else if (az >= nz - 1) { a[0] = ar + (int64_t)az * nr; b[0] = 1; }
    else {
      a[0] = ar + (int64_t)az * nr; a[2] = ar + (int64_t)(az + 1) * nr;
      b[0] = ((az + 1.5) * dz - z0) / (dz);
      b[2] = (z0 - (az + 0.5) * dz) / (dz);
    }
  } else {
    if (az < 0) {
      a[2] = ar + (int64_t)(az + 1) * nr; a[3] = (ar + 1) + (int64_t)(az + 1) * nr;
      b[2] = ((ar + 1.5) * dr - r0) / (dr);
      b[3] = (r0 - (ar + 0.5) * dr) / (dr);
    } else if (az >= nz - 1) {
      a[0] = ar + (int64_t)az * nr; a[1] = (ar + 1) + (int64_t)az * nr;
      b[0] = ((ar + 1.5) * dr - r0) / (dr);
      b[1] = (r0 - (ar + 0.5) * dr) / (dr);
    } else {
      a[0] = ar + (int64_t)az * nr; a[1] = (ar + 1) + (int64_t)az * nr;
      a[2] = ar + (int64_t)(az + 1) * nr; a[3] = (ar + 1) + (int64_t)(az + 1) * nr;
      b[0] = ((ar + 1.5) * dr - r0) * ((az + 1.5) * dz - z0) / (dr * dz);
      b[1] = (r0 - (ar + 0.5) * dr) * ((az + 1.5) * dz - z0) / (dr * dz);
      b[2] = ((ar + 1.5) * dr - r0) * (z0 - (az + 0.5) * dz) / (dr * dz);
      b[3] = (r0 - (ar + 0.5) * dr) * (z0 - (az + 0.5) * dz) / (dr * dz);
    }
  }
}

static inline double shell_volume(int ar, double dr, double dz, double PHIp) {
  /* EM7.cu:175-176 */
  return PHIp / 2 * ((((ar + 1) * dr) * ((ar + 1) * dr) - (ar * dr) * (ar * dr)) * dz);
}

static void em7_one(double r0, double z0, double q, double vr, double vz, double *jr, double *jz,
                    int nr, int nz, double dr, double dz, double FN, double PHIp) {
  int64_t a[4]; double b[4]; int ar;
  em7_weights(r0, z0, nr, nz, dr, dz, a, b, &ar);
  double V1 = shell_volume(ar, dr, dz, PHIp), V2 = shell_volume(ar + 1, dr, dz, PHIp);
  const double V[4] = {V1, V2, V1, V2};
  for (int k = 0; k < 4; ++k) {                           /* EM7.cu:178-202 */
    jr[a[k]] += FN * b[k] * q * vr / V[k];
    jz[a[k]] += FN * b[k] * q * vz / V[k];
  }
}

void orc_em7(const double *r, const double *z, const double *q, const double *vr,
             const double *vz, double *jr, double *jz, const int *del, int64_t n,
             int nr, int nz, double dr, double dz, double FN, double PHIp) {
  for (int64_t i = 0; i < n; ++i) {
    if (del[i] == 1) continue;        /* EM7.cu:163-173: zero weights */
    em7_one(r[i], z[i], q[i], vr[i], vz[i], jr, jz, nr, nz, dr, dz, FN, PHIp);
  }
}

/* ================================================================= FDTD */
/* EM3_1.cu:89-95: Faraday update of H_phi (n_r x n_z), in place. */
void orc_em3_1(double *Er, double *Ez, double *H, int nr, int nz, double mu, double dr,
               double dz, double dt) {
#pragma omp parallel for schedule(static) num_threads(g_threads)
  for (int j = 0; j < nz; ++j)
    for (int i = 0; i < nr; ++i) {
      int64_t nr_ = i + (int64_t)j * nr, nz_ = i + (int64_t)j * (nr + 1);
      H[nr_] = H[nr_] + (dt / (mu * dr) * (Ez[nz_ + 1] - Ez[nz_]) -
                         dt / (mu * dz) * (Er[nr_ + nr] - Er[nr_]));
    }
}

/* EM3.cu:121-149: Ampere update, Jacobi (reads Er0/Ez0/H0, writes Er/Ez). */
void orc_em3(const double *Er0, const double *Ez0, const double *H0, double *Er, double *Ez,
             const double *jr, const double *jz, int nr, int nz, double eps, double dr,
             double dz, double dt, unsigned flags) {
#pragma omp parallel for schedule(static) num_threads(g_threads)
  for (int j = 0; j <= nz; ++j) {
    for (int i = 0; i <= nr; ++i) {
      int64_t n_r = i + (int64_t)j * nr, n_z = i + (int64_t)j * (nr + 1);
      if (i < nr) {
        if (j < 1) {
          Er[n_r] = (flags & GASATT_Q_ER_END_COPY) ? Er0[n_r + nr] : 0.0;
        } else if (j >= nz) {
          Er[n_r] = (flags & GASATT_Q_ER_END_COPY) ? Er0[n_r - nr] : 0.0;
        } else {
          Er[n_r] = Er0[n_r] - dt / eps * (jr[n_r - nr] + jr[n_r]) / 2 -
                    dt / (eps * dz) * (H0[n_r] - H0[n_r - nr]);
        }
      }
      if (j < nz) {
        if (i < 1) {
          double jterm = (flags & GASATT_Q_EZ_AXIS_JSIGN) ? dt / eps * jz[n_r] : -(dt / eps * jz[n_r]);
          Ez[n_z] = Ez0[n_z] + jterm + 4 * dt / (eps * dr) * H0[n_r];
        } else if (i < nr) {
          double ri = (flags & GASATT_Q_EZ_RSHIFT) ? (i + 1) * dr : i * dr;
          Ez[n_z] = Ez0[n_z] - dt / eps * (jz[n_r - 1] + jz[n_r]) / 2 +
                    dt / eps * (1 / (2 * ri) + 1 / dr) * H0[n_r] +
                    dt / eps * (1 / (2 * ri) - 1 / dr) * H0[n_r - 1];
        } else {
          Ez[n_z] = Ez0[n_z];       /* r = Rp: never written (EM3.cu:145) */
        }
      }
    }
  }
}

/* ================================================================ EM4 */
/* EM4.cu:41-122: staggered bilinear gather with one-sided edges.  The only
 * change: the row/column index is clamped at z = Lp / r = Rp exactly, where
 * the reference reads one element past the array with weight 0. */
static void gather(const double *Er, const double *Ez, const double *H, int nr, int nz,
                   double dr, double dz, double r0, double z0, double *E_r, double *E_z,
                   double *Hp) {
  int ar, az;
  int64_t a1, a2, a3, a4;
  /* Er */
  ar = (int)floor(r0 / dr - 0.5);
  az = (int)floor(z0 / dz);
  if (az > nz - 1) az = nz - 1;
  a1 = ar + (int64_t)az * nr; a2 = (ar + 1) + (int64_t)az * nr;
  a3 = ar + (int64_t)(az + 1) * nr; a4 = (ar + 1) + (int64_t)(az + 1) * nr;
  if (ar < 0) *E_r = (Er[a2] * (az * dz + dz - z0) + Er[a4] * (z0 - az * dz)) / dz;
  else if (ar >= nr - 1) *E_r = (Er[a1] * (az * dz + dz - z0) + Er[a3] * (z0 - az * dz)) / dz;
  else
    *E_r = (Er[a1] * ((ar + 1.5) * dr - r0) * ((az + 1) * dz - z0) +
            Er[a2] * (r0 - (ar + 0.5) * dr) * ((az + 1) * dz - z0) +
            Er[a3] * ((ar + 1.5) * dr - r0) * (z0 - az * dz) +
            Er[a4] * (r0 - (ar + 0.5) * dr) * (z0 - az * dz)) / (dr * dz);
  /* Ez */
  ar = (int)floor(r0 / dr);
  az = (int)floor(z0 / dz - 0.5);
  if (ar > nr - 1) ar = nr - 1;
  a1 = ar + (int64_t)az * (nr + 1); a2 = (ar + 1) + (int64_t)az * (nr + 1);
  a3 = ar + (int64_t)(az + 1) * (nr + 1); a4 = (ar + 1) + (int64_t)(az + 1) * (nr + 1);
  if (az < 0) *E_z = (Ez[a3] * (ar * dr + dr - r0) + Ez[a4] * (r0 - ar * dr)) / dr;
  else if (az >= nz - 1) *E_z = (Ez[a1] * (ar * dr + dr - r0) + Ez[a2] * (r0 - ar * dr)) / dr;
  else
    *E_z = (Ez[a1] * ((ar + 1) * dr - r0) * ((az + 1.5) * dz - z0) +
            Ez[a2] * (r0 - ar * dr) * ((az + 1.5) * dz - z0) +
            Ez[a3] * ((ar + 1) * dr - r0) * (z0 - (az + 0.5) * dz) +
            Ez[a4] * (r0 - ar * dr) * (z0 - (az + 0.5) * dz)) / (dr * dz);
  /* Hphi */
  ar = (int)floor(r0 / dr - 0.5);
  az = (int)floor(z0 / dz - 0.5);
  a1 = ar + (int64_t)az * nr; a2 = (ar + 1) + (int64_t)az * nr;
  a3 = ar + (int64_t)(az + 1) * nr; a4 = (ar + 1) + (int64_t)(az + 1) * nr;
  if (ar < 0) {
    if (az < 0) *Hp = H[a4];
    else if (az >= nz - 1) *Hp = H[a2];
    else *Hp = (H[a2] * ((az + 1.5) * dz - z0) + H[a4] * (z0 - (az + 0.5) * dz)) / dz;
  } else if (ar >= nr - 1) {
    if (az < 0) *Hp = H[a3];
    else if (az >= nz - 1) *Hp = H[a1];
    else *Hp = (H[a1] * ((az + 1.5) * dz - z0) + H[a3] * (z0 - (az + 0.5) * dz)) / dz;
  } else if (az < 0) {
    *Hp = (H[a3] * ((ar + 1.5) * dr - r0) + H[a4] * (r0 - (ar + 0.5) * dr)) / dr;
  } else if (az >= nz - 1) {
    *Hp = (H[a1] * ((ar + 1.5) * dr - r0) + H[a2] * (r0 - (ar + 0.5) * dr)) / dr;
  } else {
    *Hp = (H[a1] * ((ar + 1.5) * dr - r0) * ((az + 1.5) * dz - z0) +
           H[a2] * (r0 - (ar + 0.5) * dr) * ((az + 1.5) * dz - z0) +
           H[a3] * ((ar + 1.5) * dr - r0) * (z0 - (az + 0.5) * dz) +
           H[a4] * (r0 - (ar + 0.5) * dr) * (z0 - (az + 0.5) * dz)) / (dr * dz);
  }
}

/* relativistic Boris rotation for u = gamma v (corrected push) */
static void boris(double *ux, double *uy, double *uz, double Ex, double Ey, double Ez,
                  double Bx, double By, double Bz, double qm_dt2, double c) {
  double umx = *ux + qm_dt2 * Ex, umy = *uy + qm_dt2 * Ey, umz = *uz + qm_dt2 * Ez;
  double gm = sqrt(1 + (umx * umx + umy * umy + umz * umz) / (c * c));
  double f = qm_dt2 / gm;
  double tx = f * Bx, ty = f * By, tz = f * Bz;
  double t2 = tx * tx + ty * ty + tz * tz;
  double upx = umx + (umy * tz - umz * ty);
  double upy = umy + (umz * tx - umx * tz);
  double upz = umz + (umx * ty - umy * tx);
  double s = 2 / (1 + t2);
  double sx = s * tx, sy = s * ty, sz = s * tz;
  double wx = umx + (upy * sz - upz * sy);
  double wy = umy + (upz * sx - upx * sz);
  double wz = umz + (upx * sy - upy * sx);
  *ux = wx + qm_dt2 * Ex; *uy = wy + qm_dt2 * Ey; *uz = wz + qm_dt2 * Ez;
}

/* EM4.cu:36-177 */
void orc_em4(double *x, double *y, double *z, double *vx, double *vy, double *vz,
             double *r, double *phi, const double *vr, const double *Er, const double *Ez,
             const double *H, const double *q, const double *m, double *E, int *del,
             int64_t n, double Rp, double Lp, double PHIp, int nr, int nz,
             double mu, double c, double dr, double dz, double dt, unsigned flags) {
  for (int64_t i = 0; i < n; ++i) {
    if (del[i] == 1) continue;
    double Er0, Ez0, H0;
    gather(Er, Ez, H, nr, nz, dr, dz, r[i], z[i], &Er0, &Ez0, &H0);
    double gamma, ux, uy, uz;
    gamma = 1 / sqrt(1 - (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]) / (c * c));
    if (flags & GASATT_Q_EULER_KICK) {
      double Fr = q[i] * (Er0 + (-vz[i] * H0 * mu));        /* EM4.cu:126-129 */
      double Fz = q[i] * (Ez0 + (vr[i] * H0 * mu));
      double Fx = Fr * cos(phi[i]), Fy = Fr * sin(phi[i]);
      ux = gamma * vx[i] + Fx / m[i] * dt;                  /* EM4.cu:134-137 */
      uy = gamma * vy[i] + Fy / m[i] * dt;
      uz = gamma * vz[i] + Fz / m[i] * dt;
    } else {
      double cp = cos(phi[i]), sp = sin(phi[i]);
      ux = gamma * vx[i]; uy = gamma * vy[i]; uz = gamma * vz[i];
      double B = mu * H0;
      boris(&ux, &uy, &uz, Er0 * cp, Er0 * sp, Ez0, -B * sp, B * cp, 0.0,
            q[i] / m[i] * dt / 2, c);
    }
    gamma = sqrt(1 + (ux * ux + uy * uy + uz * uz) / (c * c));   /* EM4.cu:138 */
    E[i] = (gamma - 1) * m[i] * c * c;
    vx[i] = ux / gamma; vy[i] = uy / gamma; vz[i] = uz / gamma;
    halfdrift_cart(&x[i], &y[i], &z[i], &vx[i], &vy[i], &vz[i], vx[i], vy[i], vz[i],
                   &r[i], &phi[i], &del[i], Rp, Lp, PHIp, dt, flags);
  }
}

/* ================================================================= rotate */
/* electron_transport.cu:124-137 (rotate.m:1-13 with threshold 1e-4) */
/* ref_form: perpendicular speed^2 as v*v - vz*vz (the reference's
 * expression) instead of vx*vx + vy*vy (no cancellation). */
static void rotate_v(double *vx, double *vy, double *vz, double th, double ph, int ref_form) {
  double v = sqrt(*vx * *vx + *vy * *vy + *vz * *vz);
  double p2 = ref_form ? v * v - *vz * *vz : *vx * *vx + *vy * *vy;
  double x0, y0, z0;
  if (p2 > 0.0001) {
    double s = sqrt(p2);
    x0 = *vx * cos(th) + sin(th) / s * (*vx * *vz * cos(ph) - v * *vy * sin(ph));
    y0 = *vy * cos(th) + sin(th) / s * (*vy * *vz * cos(ph) + v * *vx * sin(ph));
    z0 = *vz * cos(th) - s * sin(th) * cos(ph);
  } else {
    x0 = v * sin(th) * cos(ph);
    y0 = v * sin(th) * sin(ph);
    z0 = v * cos(th);
  }
  *vx = x0; *vy = y0; *vz = z0;
}

/* ====================================================== MCC (drop-in kernel) */
static inline double pdf_k(const double *V, int ne, int i, int k, double a0, double b0,
                           double TCS, double pi) {
  int64_t i1 = (int64_t)i * 181 + k, i2 = (int64_t)(i + 1) * 181 + k;
  const int64_t last = (int64_t)ne * 181 - 1;
  if (i1 > last) i1 = last;
  if (i2 > last) i2 = last;
  double vI = a0 * V[i1] + b0 * V[i2];
  double D = exp(vI);
  D = 2 * pi * sin(k * pi / 180) * D * 2;
  return 1 / TCS * D;
}

/* elastic polar angle, electron_transport.cu:88-121 (flags GASATT_Q_XS_LINEAR_E,
 * GASATT_Q_CDF_NEXTBIN) or get_ElasticSc_sub1.m:4-19 (cumtrapz, interp1) */
static double elastic_theta(double energy, const double *xI, const double *yI, const double *V,
                            int ne, double U, double pi, unsigned flags) {
  double Ee = (flags & GASATT_Q_XS_LINEAR_E) ? energy : log(energy);
  if (!(flags & GASATT_Q_XS_LINEAR_E)) {
    if (Ee < xI[0]) Ee = xI[0];
    if (Ee > xI[ne - 1]) Ee = xI[ne - 1];
  }
  int i = 0;
  while (i < ne - 2 && Ee > xI[i + 1]) i++;
  double a0 = (xI[i + 1] - Ee) / (xI[i + 1] - xI[i]);
  double b0 = (Ee - xI[i]) / (xI[i + 1] - xI[i]);
  double TCS = (a0 * yI[i] + b0 * yI[i + 1]) * 2;
  if (flags & GASATT_Q_CDF_NEXTBIN) {
    double imax = 0;
    for (int k = 0; k <= 180; ++k) imax = imax + pdf_k(V, ne, i, k, a0, b0, TCS, pi) * pi / 180;
    double rnd = U * imax;
    double i1 = 0;
    int k = 0;
    while (rnd > i1 && k < 181) {
      i1 = i1 + pdf_k(V, ne, i, k, a0, b0, TCS, pi) * pi / 180;
      k++;
    }
    double i2 = i1 + pdf_k(V, ne, i, k, a0, b0, TCS, pi) * pi / 180;
    double aa = (i2 - rnd) / (i2 - i1), bb = (rnd - i1) / (i2 - i1);
    return (aa * (k - 1) + bb * k) * pi / 180;
  }
  double pdf[181], C[181];
  for (int k = 0; k <= 180; ++k) pdf[k] = pdf_k(V, ne, i, k, a0, b0, TCS, pi);
  C[0] = 0;
  const double h = pi / 180;
  for (int k = 1; k <= 180; ++k) C[k] = C[k - 1] + (pdf[k - 1] + pdf[k]) / 2 * h;
  double rn = U * C[180];
  int lo = 0, hi = 180;
  while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (C[mid] <= rn) lo = mid; else hi = mid; }
  return (lo + (rn - C[lo]) / (C[lo + 1] - C[lo])) * h;
}

static inline double powf_or_pow(double a, double b, unsigned flags) {
  if (flags & GASATT_Q_EXC_POWF) return (double)powf((float)a, (float)b);
  return pow(a, b);
}

/* mean excitation energy loss [eV]: electron_transport.cu:207-219, get_ImpExc2.m */
static double exc_loss(double T, const double *t_exc, int n_exc, unsigned flags, int *ok) {
  double k1 = 0, k2 = 0;
  for (int i = 0; i < n_exc; ++i) {
    double k = t_exc[i], A = t_exc[n_exc + i], om = t_exc[2 * n_exc + i];
    double nu = t_exc[3 * n_exc + i], ga = t_exc[4 * n_exc + i];
    if (!(flags & GASATT_Q_EXC_POWF) && !(T > k)) continue;
    double a = GASATT_MCC_Q0 * A / (k * k);
    double b = powf_or_pow(k / T, om, flags);
    double c = powf_or_pow(powf_or_pow(1 - k / T, ga, flags), nu, flags);
    k1 = k1 + a * b * c * k;
    k2 = k2 + a * b * c;
  }
  *ok = k2 != 0;
  return k1 / k2;
}

void orc_electron_transport(double *x, double *y, double *z, double *vx, double *vy, double *vz,
                            const double *sig_el, const double *sig_ion, const double *sig_exc,
                            const double *energy, const double *xI, const double *yI,
                            const double *V, int ne, const double *density,
                            const double *temperature, int64_t ncell, const double *dphi,
                            const double *t_exc, int n_exc, uint8_t *sec, double *svx,
                            double *svy, double *svz, double *sample_out, double *ivx,
                            double *ivy, double *ivz, const int *sum_cell0, int rmax,
                            int cellnumxy, double dr, double dz, double dt, int64_t n,
                            const double *draws, unsigned flags) {
  (void)z;
  const double e = GASATT_MCC_E, c = GASATT_MCC_C, m = GASATT_MCC_ME, m_ion = GASATT_MCC_MION;
  const double kb = GASATT_MCC_KB, E_e = m * c * c / e;
  const double pi = (flags & GASATT_Q_PI7) ? GASATT_MCC_PI7 : GASATT_PI;
  const double I = GASATT_ION_I_EV;
  for (int64_t p = 0; p < n; ++p) {
    const double *U = draws + p * GASATT_MCC_NDRAW;
    double v_e = sqrt(vx[p] * vx[p] + vy[p] * vy[p] + vz[p] * vz[p]);   /* :64-65 */
    double dx = v_e * dt;
    double r = sqrt(x[p] * x[p] + y[p] * y[p]);                         /* :67-72 */
    double phi = atan(y[p] / x[p]);
    int iz = (int)floor(z[p] / dz), ir = (int)floor(r / dr);
    if (ir > rmax - 1) ir = rmax - 1;
    if (ir < 0) ir = 0;
    int iphi = (int)floor(phi / dphi[ir]);
    int nphi = sum_cell0[ir + 1] - sum_cell0[ir];
    if (iphi > nphi - 1) iphi = nphi - 1;
    if (iphi < 0) iphi = 0;
    int64_t index = (int64_t)iz * cellnumxy + sum_cell0[ir] + iphi;
    if (index < 0) index = 0;
    if (index > ncell - 1) index = ncell - 1;
    double p_el = dx * density[index] * sig_el[p];                      /* :74-79 */
    double p_io = dx * density[index] * sig_ion[p];
    double p_ex = dx * density[index] * sig_exc[p];
    double p_tot = p_el + p_io + p_ex;
    double a = p_el / p_tot;
    double b = a + p_io / p_tot;
    if (!(flags & GASATT_Q_COLL_LINEAR_P)) p_tot = -expm1(-p_tot);
    double p1 = U[0], p2 = U[1];
    if (!(p1 < p_tot)) continue;
    if (p2 < a) {                                                        /* :86-137 */
      double th = elastic_theta(energy[p], xI, yI, V, ne, U[2], pi, flags);
      double ph = 2 * pi * U[3];
      rotate_v(&vx[p], &vy[p], &vz[p], th, ph, 1);
    } else if (p2 < b && energy[p] > I / 1000) {                         /* :139-205 */
      double T = energy[p] * 1000;
      double T_a = 1000, T_b = 2 * I, t_b = I, T_s = 4.17, t_s = 13.8;
      double T_0 = T_s - T_a / (T + T_b);
      double t = t_s * T / (T + t_b);
      double T_m = (T - I) / 2;
      double Rn = U[2];
      double k_1 = atan((T_m - T_0) / t);
      double k_2 = atan(T_0 / t);
      double k0 = T_0 + t * tan(Rn * (k_1 + k_2) - k_2);
      double E_1 = k0, E_2 = T - E_1 - I, E_p, E_s;
      if (E_2 > E_1) { E_p = E_2; E_s = E_1; } else { E_p = E_1; E_s = E_2; }
      double kk = (flags & GASATT_Q_SEC_LAB_FRAME) ? k0 : E_s;
      E_p = E_p * e;
      E_s = E_s * e;
      double phi_p = 2 * pi * U[3];
      double phi_s = phi_p - pi;
      double sin_tp = sqrt((kk / T) / ((1 - kk / T) * T / (2 * E_e) + 1));
      double th_p = asin(sin_tp);
      double sin_ts = sqrt((1 - kk / T) / (1 + kk / (2 * E_e)));
      double th_s = asin(sin_ts);
      double ix = vx[p] / v_e, iy = vy[p] / v_e, iz_ = vz[p] / v_e;   /* incident direction */
      double gamma = 1 + E_p / (m * c * c);
      double v_p = c * sqrt(1 - 1 / (gamma * gamma));
      double ratio = v_p / v_e;
      vx[p] = ratio * vx[p]; vy[p] = ratio * vy[p]; vz[p] = ratio * vz[p];
      rotate_v(&vx[p], &vy[p], &vz[p], th_p, phi_p, 1);
      gamma = 1 + E_s / (m * c * c);
      double v_s = c * sqrt(1 - 1 / (gamma * gamma));
      sec[p] = 1;
      if (flags & GASATT_Q_SEC_LAB_FRAME) {
        svx[p] = v_s * sin(th_s) * cos(phi_s);
        svy[p] = v_s * sin(th_s) * sin(phi_s);
        svz[p] = v_s * cos(th_s);
      } else {
        double sx = ix * v_s, sy = iy * v_s, sz = iz_ * v_s;
        rotate_v(&sx, &sy, &sz, th_s, phi_s, 1);
        svx[p] = sx; svy[p] = sy; svz[p] = sz;
      }
      sample_out[p] = (double)index;
      double sd = sqrt(m_ion / (kb * temperature[index]));
      ivx[p] = (double)(float)U[4] / sd;
      ivy[p] = (double)(float)U[5] / sd;
      ivz[p] = (double)(float)U[6] / sd;
    } else {                                                             /* :206-227 */
      double T = energy[p] * 1000;
      int ok;
      double E_dep = exc_loss(T, t_exc, n_exc, flags, &ok);
      if (!ok) continue;
      double E_p = T - E_dep;
      double gamma = 1 + E_p * e / (m * c * c);
      double v_p = c * sqrt(1 - 1 / (gamma * gamma));
      double ratio = v_p / v_e;
      vx[p] = ratio * vx[p]; vy[p] = ratio * vy[p]; vz[p] = ratio * vz[p];
    }
  }
}

/* ========================================================= MATLAB drop-ins */
void orc_free_motion(const double *vx, const double *vy, const double *vz, const double *x,
                     const double *y, const double *z, int64_t n, double dt, double *xn,
                     double *yn, double *zn, double *rn, double *phin) {
  for (int64_t i = 0; i < n; ++i) {                      /* free_motion.m:3-7 */
    xn[i] = x[i] + vx[i] * dt;
    yn[i] = y[i] + vy[i] * dt;
    zn[i] = z[i] + vz[i] * dt;
    rn[i] = sqrt(xn[i] * xn[i] + yn[i] * yn[i]);
    phin[i] = atan2(yn[i], xn[i]);
  }
}

/* REBOND.m:6-66: an azimuth below 0 is raised by PHIp, and (v1, v2) turned
 * by +PHIp, until it is not (:7-22); the wrapped particles' x, y are rebuilt
 * from r and the new azimuth (:24-25); the same downwards above PHIp
 * (:31-48); then specular reflection at z = Lp (:53-60) and at z = 0
 * (:62-67).  Every wrap and reflection counts one boundary event. */
int64_t orc_rebond(double *pos, int64_t ldp, const double *r, const double *phi, double *vel,
                   int64_t ldv, int64_t n, double Lp, double PHIp, int max_wraps) {
  const double cP = cos(PHIp), sP = sin(PHIp);
  int64_t events = 0;
  for (int64_t i = 0; i < n; ++i) {
    double ph = phi[i], v1 = vel[i], v2 = vel[ldv + i];
    int k = 0;
    if (ph < 0) {
      while (ph < 0) {
        if (++k > max_wraps) return -1;
        ph = ph + PHIp;
        const double w = v1 * cP - v2 * sP;
        v2 = v1 * sP + v2 * cP;
        v1 = w;
      }
      pos[i] = r[i] * cos(ph);
      pos[ldp + i] = r[i] * sin(ph);
    }
    if (ph > PHIp) {
      while (ph > PHIp) {
        if (++k > max_wraps) return -1;
        ph = ph - PHIp;
        const double w = v1 * cP + v2 * sP;
        v2 = -v1 * sP + v2 * cP;
        v1 = w;
      }
      pos[i] = r[i] * cos(ph);
      pos[ldp + i] = r[i] * sin(ph);
    }
    vel[i] = v1;
    vel[ldv + i] = v2;
    double z = pos[2 * ldp + i], vz = vel[2 * ldv + i];
    if (z > Lp) { z = 2 * Lp - z; vz = -vz; ++k; }
    if (z < 0) { z = -z; vz = -vz; ++k; }
    pos[2 * ldp + i] = z;
    vel[2 * ldv + i] = vz;
    events += k;
  }
  return events;
}

/* particle_density.m:24-34: round(x/d + 0.5) indices (MATLAB round = half
 * away from zero), sparse histogram, FN / VC. */
void orc_particle_density(double dr, double dz, const double *dphi, int rmax, const double *r,
                          const double *phi, const double *z, int64_t n, int cellnumxy,
                          const double *sum_cell, const double *VC, int64_t ncell, double FN,
                          double *density) {
  for (int64_t c = 0; c < ncell; ++c) density[c] = 0;
  for (int64_t i = 0; i < n; ++i) {
    double iz = round(z[i] / dz + 0.5), ir = round(r[i] / dr + 0.5);
    if (!(ir >= 1 && ir <= rmax)) continue;
    double ip = round(phi[i] / dphi[(int)ir - 1] + 0.5);
    double base = ((int)ir != 1) ? sum_cell[(int)ir - 2] : 0.0;
    double idx = (iz - 1) * cellnumxy + base + ip;
    if (!(idx >= 1 && idx <= (double)ncell)) continue;
    density[(int64_t)idx - 1] += 1.0;
  }
  for (int64_t c = 0; c < ncell; ++c) density[c] = FN * density[c] / VC[c % cellnumxy];
}

int orc_electricmagneticfield6(double *e_pos, double *e_vel, int64_t n_e, double *i1_pos,
                               double *i1_vel, int64_t n_i1, double *i2_pos, double *i2_vel,
                               int64_t n_i2, double *Er, double *Ez, double *H, int nr, int nz,
                               double delta, double dt, double Rp, double Lp, double PHIp,
                               double FN, int cycle_time, double *kin, int64_t *n_e_out,
                               int64_t *n_i1_out, int64_t *n_i2_out, unsigned flags) {
  const double e = GASATT_EM_E, m_e = GASATT_EM_ME, m_i = GASATT_EM_MION, c = GASATT_EM_C;
  const double eps = GASATT_EM_EPS, mu = GASATT_EM_MU;
  const double dr = delta, dz = delta;
  const int64_t N = n_e + n_i1 + n_i2;
  double *buf = (double *)calloc((size_t)(N > 0 ? N : 1) * 13, sizeof(double));
  int *del = (int *)calloc((size_t)(N > 0 ? N : 1), sizeof(int));
  double *x = buf, *y = x + N, *z = y + N, *vx = z + N, *vy = vx + N, *vz = vy + N;
  double *r = vz + N, *phi = r + N, *vr = phi + N, *q = vr + N, *m = q + N, *E = m + N;
  double *pos[3] = {e_pos, i1_pos, i2_pos}, *vel[3] = {e_vel, i1_vel, i2_vel};
  const int64_t cnt[3] = {n_e, n_i1, n_i2};
  const double qs[3] = {-e, e, 2 * e}, ms[3] = {m_e, m_i, m_i};   /* :68-69 */
  int64_t o = 0;
  for (int s = 0; s < 3; ++s)
    for (int64_t i = 0; i < cnt[s]; ++i, ++o) {
      double p0 = pos[s][i], p1 = pos[s][cnt[s] + i], p2 = pos[s][2 * cnt[s] + i];
      if (flags & GASATT_POS_IN_CYL) { x[o] = p0 * cos(p1); y[o] = p0 * sin(p1); }  /* :113-115 */
      else { x[o] = p0; y[o] = p1; }
      z[o] = p2;
      vx[o] = vel[s][i]; vy[o] = vel[s][cnt[s] + i]; vz[o] = vel[s][2 * cnt[s] + i];
      q[o] = qs[s]; m[o] = ms[s];
    }
  const int64_t ncel = (int64_t)nr * nz;
  double *jr = (double *)calloc((size_t)ncel, sizeof(double));
  double *jz = (double *)calloc((size_t)ncel, sizeof(double));
  double *Er0 = (double *)malloc((size_t)nr * (nz + 1) * sizeof(double));
  double *Ez0 = (double *)malloc((size_t)(nr + 1) * nz * sizeof(double));
  const int ratio = 5;
  const double ddt = ratio * dt;                                        /* :134-135 */
  const int steps = cycle_time / ratio;
  for (int k = 0; k < steps; ++k) {                                     /* :138-166 */
    orc_em2(x, y, z, vx, vy, vz, r, phi, vr, del, N, Rp, Lp, PHIp, ddt, flags);
    memset(jr, 0, (size_t)ncel * sizeof(double));
    memset(jz, 0, (size_t)ncel * sizeof(double));
    orc_em7(r, z, q, vr, vz, jr, jz, del, N, nr, nz, dr, dz, FN, PHIp);
    orc_em3_1(Er, Ez, H, nr, nz, mu, dr, dz, -dt / 4);
    for (int i = 0; i < 2 * ratio; ++i) {
      orc_em3_1(Er, Ez, H, nr, nz, mu, dr, dz, dt / 2);
      memcpy(Er0, Er, (size_t)nr * (nz + 1) * sizeof(double));
      memcpy(Ez0, Ez, (size_t)(nr + 1) * nz * sizeof(double));
      orc_em3(Er0, Ez0, H, Er, Ez, jr, jz, nr, nz, eps, dr, dz, dt / 2, flags);
    }
    orc_em3_1(Er, Ez, H, nr, nz, mu, dr, dz, dt / 4);
    orc_em4(x, y, z, vx, vy, vz, r, phi, vr, Er, Ez, H, q, m, E, del, N, Rp, Lp, PHIp, nr, nz,
            mu, c, dr, dz, ddt, flags);
  }
  /* :168-188, with each species compacted by its own delete flags */
  int64_t outs[3] = {0, 0, 0};
  o = 0;
  for (int s = 0; s < 3; ++s) {
    int64_t w = 0;
    for (int64_t i = 0; i < cnt[s]; ++i, ++o) {
      if (del[o]) continue;
      pos[s][w] = x[o]; pos[s][cnt[s] + w] = y[o]; pos[s][2 * cnt[s] + w] = z[o];
      vel[s][w] = vx[o]; vel[s][cnt[s] + w] = vy[o]; vel[s][2 * cnt[s] + w] = vz[o];
      if (s == 0) kin[w] = E[o] / (1000 * e);
      ++w;
    }
    outs[s] = w;
  }
  *n_e_out = outs[0]; *n_i1_out = outs[1]; *n_i2_out = outs[2];
  free(buf); free(del); free(jr); free(jz); free(Er0); free(Ez0);
  return 0;
}

int orc_electron_collision(double *e_pos, double *e_vel, int64_t n_e, int64_t cap_e,
                           double *i1_pos, double *i1_vel, int64_t n_i1, int64_t cap_i1,
                           const gasatt_tables *tab, const double *kin, const double *sum_cell,
                           int rmax, int cellnumxy, const double *density,
                           const double *temperature, int64_t ncell, double PHIp,
                           const double *phimax, double dr, double dz, const double *sig_el,
                           const double *sig_ion, const double *sig_exc, double dt,
                           const double *draws, int64_t *n_e_out, int64_t *n_i1_out,
                           unsigned flags) {
  double xI[64], yI[64], *V = (double *)malloc(181 * 64 * sizeof(double));
  int ne = orc_elastic_tables(tab, xI, yI, V);
  if (ne < 2 || ne > 64) { free(V); return GASATT_E_TABLES; }
  int *sc0 = (int *)malloc((size_t)(rmax + 1) * sizeof(int));
  double *dphi = (double *)malloc((size_t)rmax * sizeof(double));
  sc0[0] = 0;                                                            /* :53-54 */
  for (int i = 0; i < rmax; ++i) { sc0[i + 1] = (int)sum_cell[i]; dphi[i] = PHIp * 1 / phimax[i]; }
  const int64_t n = n_e;
  uint8_t *sec = (uint8_t *)calloc((size_t)(n > 0 ? n : 1), 1);
  double *w = (double *)calloc((size_t)(n > 0 ? n : 1) * 7, sizeof(double));
  double *svx = w, *svy = w + n, *svz = w + 2 * n, *smp = w + 3 * n, *ivx = w + 4 * n,
         *ivy = w + 5 * n, *ivz = w + 6 * n;
  orc_electron_transport(e_pos, e_pos + cap_e, e_pos + 2 * cap_e, e_vel, e_vel + cap_e,
                         e_vel + 2 * cap_e, sig_el, sig_ion, sig_exc, kin, xI, yI, V, ne,
                         density, temperature, ncell, dphi, tab->t_exc, tab->n_exc, sec, svx,
                         svy, svz, smp, ivx, ivy, ivz, sc0, rmax, cellnumxy, dr, dz, dt, n,
                         draws, flags);
  int64_t nb = 0;
  for (int64_t i = 0; i < n; ++i) nb += sec[i];
  if (n_e + nb > cap_e || n_i1 + nb > cap_i1) {
    free(V); free(sc0); free(dphi); free(sec); free(w);
    return GASATT_E_CAPACITY;
  }
  int64_t we = n_e, wi = n_i1;                                           /* :63-75 */
  for (int64_t i = 0; i < n; ++i) {
    if (!sec[i]) continue;
    for (int d = 0; d < 3; ++d) {
      i1_pos[d * cap_i1 + wi] = e_pos[d * cap_e + i];
      e_pos[d * cap_e + we] = e_pos[d * cap_e + i];
    }
    i1_vel[wi] = ivx[i]; i1_vel[cap_i1 + wi] = ivy[i]; i1_vel[2 * cap_i1 + wi] = ivz[i];
    e_vel[we] = svx[i]; e_vel[cap_e + we] = svy[i]; e_vel[2 * cap_e + we] = svz[i];
    ++we; ++wi;
  }
  *n_e_out = we; *n_i1_out = wi;
  free(V); free(sc0); free(dphi); free(sec); free(w);
  return 0;
}

/* ============================================ resident step (corrected physics) */
/* Product tables: cross-sections on G log-spaced energies (find_CS0.m with the
 * corrected out-of-table policy), normalised elastic CDFs per grid energy
 * (get_ElasticSc_sub1.m: log DCS linear in log E, PDF = 2 pi sin(theta) DCS,
 * cumtrapz), and the FP64 null-collision bound
 *   nu_max = n * max_g v(E_{g+1}) * max(sigma_tot[g], sigma_tot[g+1]),
 * an upper bound of n v(E) sigma_tot(E) under the linear-in-log-index lookup
 * (v grows with E; a linear sigma is bounded by its end values), including
 * E < E_min (sigma[0], v(E_min)) and E > E_max (sigma[G-1], v < c). */
static int xs_fill(const gasatt_tables *t, int G, double emin_ev, double emax_ev, double n_gas,
                   double c, double me, double qe, double *sig_el, double *sig_ion,
                   double *sig_exc, double *cdf, double *nu_max) {
  double xI[64], yI[64], *V = (double *)malloc(181 * 64 * sizeof(double));
  int ne = orc_elastic_tables(t, xI, yI, V);
  if (ne < 2 || ne > 64) { free(V); return GASATT_E_TABLES; }
  const double lnEmin = log(emin_ev), dl = (log(emax_ev) - lnEmin) / (G - 1);
  double *Eg = (double *)malloc((size_t)G * sizeof(double));
  for (int g = 0; g < G; ++g) {
    Eg[g] = exp(lnEmin + g * dl);
    double E_keV = Eg[g] / 1000;
    cs0_one(t, E_keV, &sig_el[g], &sig_ion[g], &sig_exc[g], 0u);
  }
  const double h = GASATT_PI / 180;
  for (int g = 0; g < G; ++g) {
    double le = log(Eg[g] / 1000);
    if (le < xI[0]) le = xI[0];
    if (le > xI[ne - 1]) le = xI[ne - 1];
    int i = 0;
    while (i < ne - 2 && le > xI[i + 1]) i++;
    double a0 = (xI[i + 1] - le) / (xI[i + 1] - xI[i]);
    double b0 = (le - xI[i]) / (xI[i + 1] - xI[i]);
    double *C = cdf + (int64_t)g * 181;
    double prev = 0;
    C[0] = 0;
    for (int k = 0; k <= 180; ++k) {
      double vI = a0 * V[(int64_t)i * 181 + k] + b0 * V[(int64_t)(i + 1) * 181 + k];
      double pdf = 2 * GASATT_PI * sin(k * h) * exp(vI) * 2;
      if (k > 0) C[k] = C[k - 1] + (prev + pdf) / 2 * h;
      prev = pdf;
    }
    double tot = C[180];
    for (int k = 0; k <= 180; ++k) C[k] = C[k] / tot;
  }
  double vmax = 0;
  for (int g = 0; g <= G; ++g) {
    double sg, vg;
    if (g == G) { sg = sig_el[G - 1] + sig_ion[G - 1] + sig_exc[G - 1]; vg = c; }
    else {
      double s0 = sig_el[g] + sig_ion[g] + sig_exc[g];
      double s1 = (g + 1 < G) ? sig_el[g + 1] + sig_ion[g + 1] + sig_exc[g + 1] : s0;
      sg = s0 > s1 ? s0 : s1;
      double Eu = (g + 1 < G) ? Eg[g + 1] : Eg[g];
      double eps_ = Eu * qe / (me * c * c);
      double gam = 1 + eps_;
      vg = c * sqrt(eps_ * (2 + eps_)) / gam;
    }
    double nv = sg * vg;
    if (nv > vmax) vmax = nv;
  }
  *nu_max = n_gas * vmax;
  free(V); free(Eg);
  return 0;
}

typedef struct pass_ctx {
  const gasatt_sim_config *cfg;
  const orc_xs *xs;
  double lnEmin, dlnE;
} pass_ctx;

static void xs_lookup(const orc_xs *xs, double Eev, double *se, double *si, double *sx, double *L_o) {
  double L = (log(Eev) - xs->lnEmin) / xs->dlnE;
  int i; double f;
  if (!(L > 0)) { i = 0; f = 0; }
  else if (L >= xs->G - 1) { i = xs->G - 2; f = 1; }
  else { i = (int)L; f = L - i; }
  *se = xs->sig_el[i] + f * (xs->sig_el[i + 1] - xs->sig_el[i]);
  *si = xs->sig_ion[i] + f * (xs->sig_ion[i + 1] - xs->sig_ion[i]);
  *sx = xs->sig_exc[i] + f * (xs->sig_exc[i + 1] - xs->sig_exc[i]);
  *L_o = L;
}

static double cdf_theta(const orc_xs *xs, double L, double U) {
  double Lr = floor(L + 0.5);
  int g = Lr < 0 ? 0 : (Lr > xs->G - 1 ? xs->G - 1 : (int)Lr);
  const double *C = xs->cdf + (int64_t)g * 181;
  int lo = 0, hi = 180;
  while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (C[mid] <= U) lo = mid; else hi = mid; }
  return (lo + (U - C[lo]) / (C[lo + 1] - C[lo])) * (GASATT_PI / 180);
}

/* mean excitation energy loss (electron_transport.cu:207-219, get_ImpExc2.m)
 * tabulated on the grid at build time and interpolated like the
 * cross-sections; *ok = 0 below the lowest threshold or for a loss outside
 * (0, T) */
static double exc_loss_sim(const orc_xs *xs, double T, double L, int *ok) {
  *ok = 0;
  if (!(T > xs->exc_kmin)) return 0;
  int i; double f;
  if (!(L > 0)) { i = 0; f = 0; }
  else if (L >= xs->G - 1) { i = xs->G - 2; f = 1; }
  else { i = (int)L; f = L - i; }
  double e = xs->edep[i] + f * (xs->edep[i + 1] - xs->edep[i]);
  *ok = (e > 0) && (e < T);
  return e;
}

static double exc_loss_exact(const orc_xs *xs, double T) {
  double k1 = 0, k2 = 0;
  for (int i = 0; i < xs->n_exc; ++i) {
    double k = xs->exc_k[i];
    if (!(T > k)) continue;
    double a = xs->exc_A[i] / (k * k);
    double b = pow(k / T, xs->exc_om[i]);
    double c = pow(1 - pow(k / T, xs->exc_ga[i]), xs->exc_nu[i]);
    k1 = k1 + a * b * c * k;
    k2 = k2 + a * b * c;
  }
  return k2 > 0 ? k1 / k2 : 0.0;
}

/* u magnitude for kinetic energy E [J]: c sqrt(eps (2 + eps)), eps = E / (m c^2) */
static inline double u_of_energy(double EJ, double m, double c) {
  double eps_ = EJ / (m * c * c);
  return c * sqrt(eps_ * (2 + eps_));
}

static void halfdrift_u(double *x, double *y, double *z, double *ux, double *uy, double *uz,
                        uint8_t *alive, const gasatt_sim_config *cfg, double Rp, double Lp) {
  double g = sqrt(1 + (*ux * *ux + *uy * *uy + *uz * *uz) / (cfg->c * cfg->c));
  double r, ph;
  int del = 0;
  halfdrift_cart(x, y, z, ux, uy, uz, *ux / g, *uy / g, *uz / g, &r, &ph, &del, Rp, Lp,
                 cfg->PHIp, cfg->dt, cfg->flags);
  if (del) *alive = 0;
}

static void deposit_u(double x, double y, double z, double ux, double uy, double uz,
                      const gasatt_sim_config *cfg, double *jr, double *jz) {
  double g = sqrt(1 + (ux * ux + uy * uy + uz * uz) / (cfg->c * cfg->c));
  double r = sqrt(x * x + y * y);
  double cp = r > 0 ? x / r : 1.0, sp = r > 0 ? y / r : 0.0;
  double vr = (ux * cp + uy * sp) / g, vz = uz / g;
  em7_one(r, z, -cfg->q_e, vr, vz, jr, jz, cfg->n_r, cfg->n_z, cfg->dr, cfg->dz, cfg->FN,
          cfg->PHIp);
}

/* births of one thread: state rows appended after the parallel loop */
typedef struct births_t {
  int64_t n, cap;
  double *st;        /* 6 per birth: x y z ux uy uz */
  uint64_t *id;
  uint8_t *alive;
} births_t;

static void births_push(births_t *b, const double s[6], uint64_t id, uint8_t alive) {
  if (b->n == b->cap) {
    b->cap = b->cap ? 2 * b->cap : 256;
    b->st = (double *)realloc(b->st, (size_t)b->cap * 6 * sizeof(double));
    b->id = (uint64_t *)realloc(b->id, (size_t)b->cap * sizeof(uint64_t));
    b->alive = (uint8_t *)realloc(b->alive, (size_t)b->cap);
  }
  memcpy(b->st + 6 * b->n, s, 6 * sizeof(double));
  b->id[b->n] = id;
  b->alive[b->n] = alive;
  b->n++;
}

/* per-thread current buffers, kept between calls */
static double *g_tj = NULL;
static size_t g_tj_len = 0;

int orc_sim_pass(const gasatt_sim_config *cfg, const orc_xs *xs, int64_t step, double *x,
                 double *y, double *z, double *ux, double *uy, double *uz, uint64_t *id,
                 uint8_t *alive, int64_t *n_io, int64_t cap, const double *Er, const double *Ez,
                 const double *H, double *jr, double *jz, int do_kick, int do_mcc,
                 const double *gas, const double *gas_T, orc_ions *ions, orc_counters *cnt) {
  const int nr = cfg->n_r, nz = cfg->n_z;
  const double Rp = nr * cfg->dr, Lp = nz * cfg->dz, c = cfg->c, me = cfg->m_e, qe = cfg->q_e;
  const double qm_dt2 = -qe / me * cfg->dt / 2;
  const double P_null = -expm1(-xs->nu_max * cfg->dt);
  const double I = GASATT_ION_I_EV;
  const int64_t ncel = (int64_t)nr * nz;
  const int nt = g_threads;
  const size_t need = (size_t)nt * 2 * (size_t)ncel;
  if (need > g_tj_len) {
    free(g_tj);
    g_tj = (double *)malloc(need * sizeof(double));
    g_tj_len = need;
  }
  births_t *bt = (births_t *)calloc((size_t)nt, sizeof(births_t));
  births_t *it = (births_t *)calloc((size_t)nt, sizeof(births_t));   /* ion births */
  const double ion_sigma = ions ? sqrt(cfg->kb * cfg->gas_temperature / cfg->m_ion) : 0.0;
  orc_counters *ct = (orc_counters *)calloc((size_t)nt, sizeof(orc_counters));
  const int64_t n0 = *n_io;
#pragma omp parallel num_threads(nt)
  {
#ifdef _OPENMP
    const int tid = omp_get_thread_num();
#else
    const int tid = 0;
#endif
    double *tjr = g_tj + (size_t)tid * 2 * ncel, *tjz = tjr + ncel;
    memset(tjr, 0, 2 * (size_t)ncel * sizeof(double));
    births_t *B = &bt[tid];
    births_t *IB = &it[tid];
    orc_counters *C = &ct[tid];
#pragma omp for schedule(static)
    for (int64_t p = 0; p < n0; ++p) {
      if (!alive[p]) continue;
      if (do_kick) {
        double r0 = sqrt(x[p] * x[p] + y[p] * y[p]);
        double cp = r0 > 0 ? x[p] / r0 : 1.0, sp = r0 > 0 ? y[p] / r0 : 0.0;
        double E_r, E_z, Hp;
        gather(Er, Ez, H, nr, nz, cfg->dr, cfg->dz, r0, z[p], &E_r, &E_z, &Hp);
        double B_ = cfg->mu0 * Hp;
        if (cfg->flags & GASATT_Q_EULER_KICK) {
          double g = sqrt(1 + (ux[p] * ux[p] + uy[p] * uy[p] + uz[p] * uz[p]) / (c * c));
          double vr = (ux[p] * cp + uy[p] * sp) / g, vz = uz[p] / g;
          double Fr = -qe * (E_r + (-vz * Hp * cfg->mu0)), Fz = -qe * (E_z + (vr * Hp * cfg->mu0));
          ux[p] += Fr * cp / me * cfg->dt; uy[p] += Fr * sp / me * cfg->dt; uz[p] += Fz / me * cfg->dt;
        } else {
          boris(&ux[p], &uy[p], &uz[p], E_r * cp, E_r * sp, E_z, -B_ * sp, B_ * cp, 0.0, qm_dt2, c);
        }
        halfdrift_u(&x[p], &y[p], &z[p], &ux[p], &uy[p], &uz[p], &alive[p], cfg, Rp, Lp);
        if (!alive[p]) { C->lost++; continue; }
      }
      halfdrift_u(&x[p], &y[p], &z[p], &ux[p], &uy[p], &uz[p], &alive[p], cfg, Rp, Lp);
      if (!alive[p]) { C->lost++; continue; }
      deposit_u(x[p], y[p], z[p], ux[p], uy[p], uz[p], cfg, tjr, tjz);
      if (do_mcc) {
        double U1, U2;
        draw_block(cfg->seed, id[p], step, 0, &U1, &U2);
        if (U1 < P_null) {
          double u2 = ux[p] * ux[p] + uy[p] * uy[p] + uz[p] * uz[p];
          double g = sqrt(1 + u2 / (c * c));
          double EJ = me * c * c * ((u2 / (c * c)) / (g + 1));
          double Eev = EJ / qe;
          double um = sqrt(u2), v = um / g;
          double se, si, sx, L;
          xs_lookup(xs, Eev, &se, &si, &sx, &L);
          double ng = cfg->gas_density, isig = ion_sigma;
          if (gas || gas_T) {
            /* density and temperature of the cell the electron ends the step in */
            double r = sqrt(x[p] * x[p] + y[p] * y[p]);
            int ir = (int)floor(r / cfg->dr), iz = (int)floor(z[p] / cfg->dz);
            ir = ir < 0 ? 0 : ir > nr - 1 ? nr - 1 : ir;
            iz = iz < 0 ? 0 : iz > nz - 1 ? nz - 1 : iz;
            if (gas) ng = gas[ir + (int64_t)iz * nr];
            if (gas_T) isig = sqrt(cfg->kb * gas_T[ir + (int64_t)iz * nr] / cfg->m_ion);
          }
          double nu_el = ng * se * v, nu_io = ng * si * v;
          double nu_ex = ng * sx * v;
          double X = U2 * xs->nu_max;
          if (X < nu_el) {
            double U3, U4;
            draw_block(cfg->seed, id[p], step, 1, &U3, &U4);
            double th = cdf_theta(xs, L, U3), ph = 2 * GASATT_PI * U4;
            rotate_v(&ux[p], &uy[p], &uz[p], th, ph, 0);
            C->ela++;
          } else if (X < nu_el + nu_io && Eev > I) {
            double U3, U4;
            draw_block(cfg->seed, id[p], step, 1, &U3, &U4);
            double T = Eev;
            double T_a = 1000, T_b = 2 * I, t_b = I, T_s = 4.17, t_s = 13.8;
            double T_0 = T_s - T_a / (T + T_b);
            double t = t_s * T / (T + t_b);
            double T_m = (T - I) / 2;
            double k_1 = atan((T_m - T_0) / t), k_2 = atan(T_0 / t);
            double k0 = T_0 + t * tan(U3 * (k_1 + k_2) - k_2);
            double E_1 = k0, E_2 = T - E_1 - I, E_p, E_s;
            if (E_2 > E_1) { E_p = E_2; E_s = E_1; } else { E_p = E_1; E_s = E_2; }
            double E_e = me * c * c / qe;
            double phi_p = 2 * GASATT_PI * U4, phi_s = phi_p - GASATT_PI;
            double th_p = asin(sqrt((E_s / T) / ((1 - E_s / T) * T / (2 * E_e) + 1)));
            double th_s = asin(sqrt((1 - E_s / T) / (1 + E_s / (2 * E_e))));
            double ix = ux[p] / um, iy = uy[p] / um, iz_ = uz[p] / um;
            double up = u_of_energy(E_p * qe, me, c), us = u_of_energy(E_s * qe, me, c);
            ux[p] = ix * up; uy[p] = iy * up; uz[p] = iz_ * up;
            rotate_v(&ux[p], &uy[p], &uz[p], th_p, phi_p, 0);
            C->ion++;
            if (ions) {
              /* Maxwellian ion: three normals by Box-Muller from draw blocks
               * 2 and 3, in the parent's local (r, theta, z) frame */
              double a1, a2, b1, b2;
              draw_block(cfg->seed, id[p], step, 2, &a1, &a2);
              draw_block(cfg->seed, id[p], step, 3, &b1, &b2);
              double ra = isig * sqrt(-2 * log(a1)), rb = isig * sqrt(-2 * log(b1));
              double wr = ra * cos(2 * GASATT_PI * a2), wt = ra * sin(2 * GASATT_PI * a2);
              double rr = sqrt(x[p] * x[p] + y[p] * y[p]);
              double cq = rr > 0 ? x[p] / rr : 1.0, sq = rr > 0 ? y[p] / rr : 0.0;
              double s[6] = {x[p], y[p], z[p], wr * cq - wt * sq, wr * sq + wt * cq,
                             rb * cos(2 * GASATT_PI * b2)};
              births_push(IB, s, orc_child_id(id[p], step), 1);
            }
            if (cfg->secondaries) {
              double s[6] = {x[p], y[p], z[p], ix * us, iy * us, iz_ * us};
              rotate_v(&s[3], &s[4], &s[5], th_s, phi_s, 0);
              births_push(B, s, orc_child_id(id[p], step), 1);
            }
          } else if (X < nu_el + nu_io + nu_ex) {
            int ok;
            double E_dep = exc_loss_sim(xs, Eev, L, &ok);
            if (ok) {
              double up = u_of_energy((Eev - E_dep) * qe, me, c);
              ux[p] = ux[p] / um * up; uy[p] = uy[p] / um * up; uz[p] = uz[p] / um * up;
              C->exc++;
              C->exc_loss_fx += llrint(E_dep * 65536.0);
            } else C->nul++;
          } else {
            C->nul++;
          }
        }
      }
    }
    /* reduce the per-thread currents in thread order */
#pragma omp for schedule(static)
    for (int64_t k = 0; k < ncel; ++k) {
      double a = 0, b = 0;
      for (int t = 0; t < nt; ++t) {
        a += g_tj[(size_t)t * 2 * ncel + k];
        b += g_tj[(size_t)t * 2 * ncel + ncel + k];
      }
      jr[k] = a;
      jz[k] = b;
    }
  }
  if (ions) {
    for (int t = 0; t < nt; ++t) {
      for (int64_t k = 0; k < it[t].n; ++k) {
        if (ions->n >= ions->cap) { ions->overflow++; continue; }
        const double *s = it[t].st + 6 * k;
        const int64_t m = ions->n++;
        ions->x[m] = s[0]; ions->y[m] = s[1]; ions->z[m] = s[2];
        ions->ux[m] = s[3]; ions->uy[m] = s[4]; ions->uz[m] = s[5];
        ions->id[m] = it[t].id[k];
        ions->alive[m] = 1;
        ions->q[m] = 1;
      }
    }
  }
  for (int t = 0; t < nt; ++t) { free(it[t].st); free(it[t].id); free(it[t].alive); }
  free(it);
  int64_t n = n0;
  for (int t = 0; t < nt; ++t) {
    cnt->ion += ct[t].ion; cnt->ela += ct[t].ela; cnt->exc += ct[t].exc;
    cnt->nul += ct[t].nul; cnt->lost += ct[t].lost;
    cnt->exc_loss_fx += ct[t].exc_loss_fx;
    for (int64_t k = 0; k < bt[t].n; ++k) {
      if (n >= cap) { cnt->cap_overflow++; continue; }
      const double *s = bt[t].st + 6 * k;
      x[n] = s[0]; y[n] = s[1]; z[n] = s[2]; ux[n] = s[3]; uy[n] = s[4]; uz[n] = s[5];
      id[n] = bt[t].id[k];
      alive[n] = bt[t].alive[k];
      ++n;
    }
    free(bt[t].st); free(bt[t].id); free(bt[t].alive);
  }
  free(bt); free(ct);
  *n_io = n;
  return 0;
}

/* The push of the resident step (kick, two half drifts, deposit) applied to
 * the ions over the ion step; electricmagneticfield6.m:68-69 pushes ion1 and
 * ion2 in the electrons' kernel with their own charge and mass. */
void orc_ion_push(const gasatt_sim_config *cfg, orc_ions *ions, const double *Er,
                  const double *Ez, const double *H, double *jr, double *jz) {
  const int nr = cfg->n_r, nz = cfg->n_z;
  const double Rp = nr * cfg->dr, Lp = nz * cfg->dz, c = cfg->c;
  const double dti = cfg->dt * cfg->ion_subcycle;
  memset(jr, 0, (size_t)nr * nz * sizeof(double));
  memset(jz, 0, (size_t)nr * nz * sizeof(double));
  for (int64_t p = 0; p < ions->n; ++p) {
    if (!ions->alive[p]) continue;
    double *x = &ions->x[p], *y = &ions->y[p], *z = &ions->z[p];
    double *ux = &ions->ux[p], *uy = &ions->uy[p], *uz = &ions->uz[p];
    const double Zq = ions->q[p];
    double r0 = sqrt(*x * *x + *y * *y);
    double cp = r0 > 0 ? *x / r0 : 1.0, sp = r0 > 0 ? *y / r0 : 0.0;
    double E_r, E_z, Hp;
    gather(Er, Ez, H, nr, nz, cfg->dr, cfg->dz, r0, *z, &E_r, &E_z, &Hp);
    double B_ = cfg->mu0 * Hp;
    boris(ux, uy, uz, E_r * cp, E_r * sp, E_z, -B_ * sp, B_ * cp, 0.0,
          Zq * cfg->q_e / cfg->m_ion * dti / 2, c);
    for (int h = 0; h < 2 && ions->alive[p]; ++h) {
      double g = sqrt(1 + (*ux * *ux + *uy * *uy + *uz * *uz) / (c * c));
      double r, ph;
      int del = 0;
      halfdrift_cart(x, y, z, ux, uy, uz, *ux / g, *uy / g, *uz / g, &r, &ph, &del, Rp, Lp,
                     cfg->PHIp, dti, cfg->flags);
      if (del) ions->alive[p] = 0;
    }
    if (!ions->alive[p]) { ions->lost++; continue; }
    double g = sqrt(1 + (*ux * *ux + *uy * *uy + *uz * *uz) / (c * c));
    double r = sqrt(*x * *x + *y * *y);
    double cq = r > 0 ? *x / r : 1.0, sq = r > 0 ? *y / r : 0.0;
    em7_one(r, *z, Zq * cfg->q_e, (*ux * cq + *uy * sq) / g, *uz / g, jr, jz, nr, nz, cfg->dr,
            cfg->dz, cfg->FN, cfg->PHIp);
  }
}

void orc_sim_fdtd(const gasatt_sim_config *cfg, double *Er, double *Ez, double *H,
                  const double *jr, const double *jz) {
  const int nr = cfg->n_r, nz = cfg->n_z, ratio = cfg->fdtd_ratio;
  const double dt = cfg->dt / ratio, mu = cfg->mu0, eps = cfg->eps0;
  double *Er0 = (double *)malloc((size_t)nr * (nz + 1) * sizeof(double));
  double *Ez0 = (double *)malloc((size_t)(nr + 1) * nz * sizeof(double));
  orc_em3_1(Er, Ez, H, nr, nz, mu, cfg->dr, cfg->dz, -dt / 4);
  for (int i = 0; i < 2 * ratio; ++i) {
    orc_em3_1(Er, Ez, H, nr, nz, mu, cfg->dr, cfg->dz, dt / 2);
    memcpy(Er0, Er, (size_t)nr * (nz + 1) * sizeof(double));
    memcpy(Ez0, Ez, (size_t)(nr + 1) * nz * sizeof(double));
    orc_em3(Er0, Ez0, H, Er, Ez, jr, jz, nr, nz, eps, cfg->dr, cfg->dz, dt / 2, cfg->flags);
  }
  orc_em3_1(Er, Ez, H, nr, nz, mu, cfg->dr, cfg->dz, dt / 4);
  free(Er0); free(Ez0);
}

/* electricmagneticfield6.m:153-154: PHIp/2 eps trapz(trapz(E^2 r)) + PHIp/2 mu trapz(trapz(H^2 r)) */
static double trapz2(const double *f, int ni, int nj, double r0, double dr, double dz, int ld) {
  double outer = 0, prev = 0;
  for (int j = 0; j < nj; ++j) {
    double inner = 0;
    for (int i = 0; i + 1 < ni; ++i) {
      double ra = r0 + i * dr, rb = r0 + (i + 1) * dr;
      double fa = f[i + (int64_t)j * ld], fb = f[i + 1 + (int64_t)j * ld];
      inner += (fa * fa * ra + fb * fb * rb) / 2 * dr;
    }
    if (j > 0) outer += (prev + inner) / 2 * dz;
    prev = inner;
  }
  return outer;
}

double orc_field_energy(const gasatt_sim_config *cfg, const double *Er, const double *Ez,
                        const double *H) {
  const int nr = cfg->n_r, nz = cfg->n_z;
  double we = trapz2(Er, nr, nz + 1, cfg->dr / 2, cfg->dr, cfg->dz, nr) +
              trapz2(Ez, nr + 1, nz, 0.0, cfg->dr, cfg->dz, nr + 1);
  double wm = trapz2(H, nr, nz, cfg->dr / 2, cfg->dr, cfg->dz, nr);
  return cfg->PHIp * 0.5 * cfg->eps0 * we + cfg->PHIp * 0.5 * cfg->mu0 * wm;
}

orc_xs *orc_xs_create(const gasatt_tables *t, int G, double emin_ev, double emax_ev,
                      double n_gas, double c, double me, double qe) {
  if (G < 2 || t->n_exc > 16) return NULL;
  orc_xs *xs = (orc_xs *)calloc(1, sizeof(orc_xs));
  xs->G = G;
  xs->lnEmin = log(emin_ev);
  xs->dlnE = (log(emax_ev) - xs->lnEmin) / (G - 1);
  xs->sig_el = (double *)malloc((size_t)G * sizeof(double));
  xs->sig_ion = (double *)malloc((size_t)G * sizeof(double));
  xs->sig_exc = (double *)malloc((size_t)G * sizeof(double));
  xs->cdf = (double *)malloc((size_t)G * 181 * sizeof(double));
  xs->edep = (double *)malloc((size_t)G * sizeof(double));
  if (xs_fill(t, G, emin_ev, emax_ev, n_gas, c, me, qe, xs->sig_el, xs->sig_ion, xs->sig_exc,
              xs->cdf, &xs->nu_max) != 0) {
    orc_xs_free(xs);
    return NULL;
  }
  xs->n_exc = t->n_exc;
  for (int i = 0; i < t->n_exc; ++i) {
    xs->exc_k[i] = t->t_exc[i];
    xs->exc_A[i] = t->t_exc[t->n_exc + i];
    xs->exc_om[i] = t->t_exc[2 * t->n_exc + i];
    xs->exc_nu[i] = t->t_exc[3 * t->n_exc + i];
    xs->exc_ga[i] = t->t_exc[4 * t->n_exc + i];
  }
  xs->exc_kmin = 1e300;
  for (int i = 0; i < t->n_exc; ++i)
    if (xs->exc_k[i] < xs->exc_kmin) xs->exc_kmin = xs->exc_k[i];
  for (int g = 0; g < G; ++g) xs->edep[g] = exc_loss_exact(xs, exp(xs->lnEmin + g * xs->dlnE));
  return xs;
}

void orc_xs_free(orc_xs *xs) {
  if (!xs) return;
  free(xs->sig_el); free(xs->sig_ion); free(xs->sig_exc); free(xs->cdf); free(xs->edep); free(xs);
}

double orc_xs_nu_max(const orc_xs *xs) { return xs->nu_max; }
const double *orc_xs_array(const orc_xs *xs, int which) {
  switch (which) {
    case 0: return xs->sig_el;
    case 1: return xs->sig_ion;
    case 2: return xs->sig_exc;
    case 4: return xs->edep;
    default: return xs->cdf;
  }
}

/* ========================================= the MATLAB CPU path (one call)
 * electricmagneticfield3.m:111-319 restated for electrons.  Constants of that
 * file (:4-11): m_e 9.1096e-31, c 3e8, eps 8.854187817e-12, mu 4 pi 1e-7,
 * e 1.6e-19.  Its REBOND calls (:113, :303) pass (position, velocity, dt, r,
 * z, phi), an older argument order than REBOND.m:1 declares; the restatement
 * applies what both mean: the azimuth atan2(y, x) wrapped into [0, PHIp] one
 * wedge at a time with (vx, vy) turned by the wedge angle and (x, y) rebuilt
 * from r and the new azimuth (REBOND.m:7-46), then z reflected at Lp and at 0
 * with vz flipped (REBOND.m:50-64). */
static const double MC_ME = 9.1096e-31, MC_C = 3e8, MC_EPS = 8.854187817e-12, MC_E = 1.6e-19;
#define MC_MU (4 * 3.141592653589793 * 1e-7)

/* half drift, wall deletion (r > R), wedge and z rules of one electron */
static void mcpu_drift(double *x, double *y, double *z, double *vx, double *vy, double vz_in,
                       double *vz_out, uint8_t *alive, double h, double R, double Lp, double PHIp) {
  double X = *x + h * *vx, Y = *y + h * *vy, Z = *z + h * vz_in, vz = vz_in;
  const double r = sqrt(X * X + Y * Y);
  if (r > R) { *alive = 0; return; }
  double ph = atan2(Y, X), v1 = *vx, v2 = *vy;
  const double cP = cos(PHIp), sP = sin(PHIp);
  if (ph < 0) {
    for (int k = 0; ph < 0 && k < 4096; ++k) {
      ph += PHIp;
      const double w = v1 * cP - v2 * sP;
      v2 = v1 * sP + v2 * cP;
      v1 = w;
    }
    X = r * cos(ph); Y = r * sin(ph);
  }
  if (ph > PHIp) {
    for (int k = 0; ph > PHIp && k < 4096; ++k) {
      ph -= PHIp;
      const double w = v1 * cP + v2 * sP;
      v2 = -v1 * sP + v2 * cP;
      v1 = w;
    }
    X = r * cos(ph); Y = r * sin(ph);
  }
  if (Z > Lp) { Z = 2 * Lp - Z; vz = -vz; }
  if (Z < 0) { Z = -Z; vz = -vz; }
  *x = X; *y = Y; *z = Z; *vx = v1; *vy = v2; *vz_out = vz;
}

/* MATLAB round (half away from zero) */
static inline double mround(double a) { return a < 0 ? -floor(-a + 0.5) : floor(a + 0.5); }

/* One axis of interp2's grids: "padded" knots 0, d/2, 3d/2, ..., L - d/2, L
 * (m cells; :221-223, :240-241) or "plain" knots 0, d, ..., m d.  Sets the
 * lower knot k and the weight t of the upper one; 0 outside (interp2 gives
 * NaN there). */
static int mcpu_axis(double q, double d, int m, int padded, int *k, double *t) {
  const double L = m * d;
  if (!(q >= 0 && q <= L)) return 0;
  if (!padded) {
    int i = (int)floor(q / d);
    if (i > m - 1) i = m - 1;
    *k = i; *t = q / d - i;
    return 1;
  }
  if (q <= d / 2) { *k = 0; *t = q / (d / 2); return 1; }
  if (q >= L - d / 2) { *k = m; *t = (q - (L - d / 2)) / (d / 2); return 1; }
  int i = (int)floor(q / d + 0.5);
  if (i < 1) i = 1;
  if (i > m - 1) i = m - 1;
  *k = i; *t = q / d + 0.5 - i;
  return 1;
}

/* value of interp2's extended grid of a field at knot (a, b) */
typedef double (*mcpu_val)(const double *F, int nr, int nz, int a, int b);
static double mc_er(const double *F, int nr, int nz, int a, int b) {   /* :224-228 */
  if (a == nr + 1) return 0.0;
  return F[(a == 0 ? 0 : a - 1) + (int64_t)b * nr];
}
static double mc_ez(const double *F, int nr, int nz, int a, int b) {   /* :232-236 */
  if (b == 0 || b == nz + 1) return 0.0;
  return F[a + (int64_t)(b - 1) * (nr + 1)];
}
static double mc_h(const double *F, int nr, int nz, int a, int b) {    /* :240-252 */
  a = a < 1 ? 1 : (a > nr ? nr : a);
  b = b < 1 ? 1 : (b > nz ? nz : b);
  return F[(a - 1) + (int64_t)(b - 1) * nr];
}
static double mcpu_interp2(const double *F, mcpu_val val, int nr, int nz, int pr, int pz,
                           double d, double r, double z) {
  int a, b;
  double tr, tz;
  if (!mcpu_axis(r, d, nr, pr, &a, &tr) || !mcpu_axis(z, d, nz, pz, &b, &tz)) return NAN;
  const double v00 = val(F, nr, nz, a, b), v10 = val(F, nr, nz, a + 1, b);
  const double v01 = val(F, nr, nz, a, b + 1), v11 = val(F, nr, nz, a + 1, b + 1);
  return (1 - tz) * ((1 - tr) * v00 + tr * v10) + tz * ((1 - tr) * v01 + tr * v11);
}

int64_t orc_mcpu_step(int64_t n, double *x, double *y, double *z, double *vx, double *vy,
                      double *vz, uint8_t *alive, double *Er, double *Ez, double *H, double *jr,
                      double *jz, int nr, int nz, double delta, double dt, double PHIp, double W) {
  const double R = nr * delta, Lp = nz * delta, d = delta;
  const int64_t ncell = (int64_t)nr * nz;
  /* :111-116 half drift, deletion, REBOND */
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t p = 0; p < n; ++p)
    if (alive[p]) mcpu_drift(&x[p], &y[p], &z[p], &vx[p], &vy[p], vz[p], &vz[p], &alive[p],
                             0.5 * dt, R, Lp, PHIp);
  /* :150-167 nearest-cell current (ind2vec), divided by W / shell volume */
  memset(jr, 0, ncell * sizeof(double));
  memset(jz, 0, ncell * sizeof(double));
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t p = 0; p < n; ++p) {
    if (!alive[p]) continue;
    const double r = sqrt(x[p] * x[p] + y[p] * y[p]);
    const double vr = vx[p] * (x[p] / r) + vy[p] * (y[p] / r);
    int ar = (int)mround(r / d + 0.5), az = (int)mround(z[p] / d + 0.5);
    ar = ar < 1 ? 1 : (ar > nr ? nr : ar);
    az = az < 1 ? 1 : (az > nz ? nz : az);
    const int64_t c = (ar - 1) + (int64_t)(az - 1) * nr;
    const double q = -MC_E;
#pragma omp atomic
    jr[c] += q * vr;
#pragma omp atomic
    jz[c] += q * vz[p];
  }
  for (int64_t c = 0; c < ncell; ++c) {
    const double Rc = (c % nr + 0.5) * d;
    const double V = PHIp * ((Rc + d / 2) * (Rc + d / 2) - (Rc - d / 2) * (Rc - d / 2)) * d;
    jr[c] = W * jr[c] / V;
    jz[c] = W * jz[c] / V;
  }
  /* :176-205 the field update: H(-dt/4), [H(dt/2), E(dt/2)] x 2, H(dt/4) */
  const int repeat = 2;
  const double dtr = dt / repeat;
  const int ldr = nr, ldz = nr + 1;
#define ER(i, j) Er[(i) + (int64_t)(j) * ldr]
#define EZ(i, j) Ez[(i) + (int64_t)(j) * ldz]
#define HH(i, j) H[(i) + (int64_t)(j) * ldr]
#define JR(i, j) jr[(i) + (int64_t)(j) * ldr]
#define JZ(i, j) jz[(i) + (int64_t)(j) * ldr]
  double *er1 = malloc(sizeof(double) * nr), *ern = malloc(sizeof(double) * nr);
  for (int sub = 0; sub <= 2 * repeat + 1; ++sub) {
    /* sub 0: H(-dtr/2); odd: H(dtr) then E(dtr); last: H(dtr/2) */
    const int last = sub == 2 * repeat + 1;
    if (sub == 0 || last || (sub & 1)) {
      const double h = sub == 0 ? -dtr / 2 : (last ? dtr / 2 : dtr);
#pragma omp parallel for num_threads(g_threads) schedule(static)
      for (int j = 0; j < nz; ++j)
        for (int i = 0; i < nr; ++i)
          HH(i, j) = HH(i, j) + h / (MC_MU * d) * (EZ(i + 1, j) - EZ(i, j)) -
                     h / (MC_MU * d) * (ER(i, j + 1) - ER(i, j));
    }
    if (!(sub & 1) || sub == 0 || last) continue;
    for (int i = 0; i < nr; ++i) { er1[i] = ER(i, 1); ern[i] = ER(i, nz - 1); }
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int j = 1; j < nz; ++j)
      for (int i = 0; i < nr; ++i)
        ER(i, j) = ER(i, j) - dtr / MC_EPS * (JR(i, j - 1) + JR(i, j)) / 2 -
                   dtr / (MC_EPS * d) * (HH(i, j) - HH(i, j - 1));
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int j = 0; j < nz; ++j) {
      for (int i = 1; i < nr; ++i) {
        const double ri = i * d;
        EZ(i, j) = EZ(i, j) - dtr / MC_EPS * (JZ(i - 1, j) + JZ(i, j)) / 2 +
                   dtr / MC_EPS * (1 / (2 * ri) + 1 / d) * HH(i, j) +
                   dtr / MC_EPS * (1 / (2 * ri) - 1 / d) * HH(i - 1, j);
      }
      EZ(0, j) = EZ(0, j) + dtr / MC_EPS * JZ(0, j) + 4 * dtr / (MC_EPS * d) * HH(0, j);
    }
    for (int i = 0; i < nr; ++i) { ER(i, 0) = er1[i]; ER(i, nz) = ern[i]; }
  }
  free(er1);
  free(ern);
#undef ER
#undef EZ
#undef HH
#undef JR
#undef JZ
  /* :216-281 interp2 gather, explicit kick; :285-319 second half drift */
  int64_t left = 0;
#pragma omp parallel for num_threads(g_threads) schedule(static) reduction(+ : left)
  for (int64_t p = 0; p < n; ++p) {
    if (!alive[p]) continue;
    const double r = sqrt(x[p] * x[p] + y[p] * y[p]);
    const double cs = x[p] / r, sn = y[p] / r;
    const double vr = vx[p] * cs + vy[p] * sn;
    const double e_r = mcpu_interp2(Er, mc_er, nr, nz, 1, 0, d, r, z[p]);
    const double e_z = mcpu_interp2(Ez, mc_ez, nr, nz, 0, 1, d, r, z[p]);
    const double h = mcpu_interp2(H, mc_h, nr, nz, 1, 1, d, r, z[p]);
    const double q = -MC_E;
    const double Fr = q * (e_r + (-vz[p] * h * MC_MU)), Fz = q * (e_z + (vr * h * MC_MU));
    const double g = 1 / sqrt(1 - (vx[p] * vx[p] + vy[p] * vy[p] + vz[p] * vz[p]) / (MC_C * MC_C));
    const double ux = g * vx[p] + Fr * cs / MC_ME * dt, uy = g * vy[p] + Fr * sn / MC_ME * dt;
    const double uz = g * vz[p] + Fz / MC_ME * dt;
    const double g2 = sqrt(1 + (ux * ux + uy * uy + uz * uz) / (MC_C * MC_C));
    vx[p] = ux / g2; vy[p] = uy / g2; vz[p] = uz / g2;
    mcpu_drift(&x[p], &y[p], &z[p], &vx[p], &vy[p], vz[p], &vz[p], &alive[p], 0.5 * dt, R, Lp, PHIp);
    left += alive[p];
  }
  return left;
}
