// gasatt_device.cuh - device helpers shared by the drop-in kernels and the
// resident simulation: counter-based RNG, staggered gather, cell-centred
// deposit weights, half drift with the reference's boundary rules, velocity
// rotation.  Formulas follow the reference kernels line by line where the
// results must agree with them (cited per function).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/gasatt.h"

namespace gasatt {

// ------------------------------------------------------------------ RNG
// Philox4x32-10 (Salmon et al., SC'11).  Counter (id_lo, id_hi, step, block),
// key = 64-bit seed.  Each block yields two (0,1) doubles from 52 bits each.
struct U2 { double a, b; };

// One Philox round: the two 32 x 32 -> 64-bit products (one wide multiply
// each) and the key mix.
__device__ __forceinline__ void philox_round(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
  const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
  const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
  c[0] = n0; c[1] = (uint32_t)p1; c[2] = n2; c[3] = (uint32_t)p0;
}

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    philox_round(c, k0, k1);
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
}

// The ten round keys of a 64-bit seed, computed once per launch on the host
// (the Weyl sequence k + i W of the key schedule), so that a kernel's rounds
// take their keys straight from its parameters.
struct PhiloxKeys {
  uint32_t k[10][2];
};

inline PhiloxKeys philox_keys(uint64_t seed) {
  PhiloxKeys K;
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  for (int i = 0; i < 10; ++i) {
    K.k[i][0] = k0; K.k[i][1] = k1;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  return K;
}

// Philox4x32-10 with the precomputed round keys (same output as philox4x32_10)
__device__ __forceinline__ void philox4x32_10(uint32_t c[4], const PhiloxKeys &K) {
#pragma unroll
  for (int i = 0; i < 10; ++i) philox_round(c, K.k[i][0], K.k[i][1]);
}

// (2b+1) 2^-53 with b the top 52 bits: exact, in (0, 1)
__device__ __forceinline__ double u01(uint32_t hi, uint32_t lo) {
  const uint64_t b = ((((uint64_t)hi) << 32) | lo) >> 12;
  return (double)b * 0x1.0p-52 + 0x1.0p-53;
}

__device__ __forceinline__ U2 draw2(uint64_t seed, uint64_t id, int64_t step, uint32_t blk) {
  uint32_t c[4] = {(uint32_t)id, (uint32_t)(id >> 32), (uint32_t)step, blk};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  return U2{u01(c[0], c[1]), u01(c[2], c[3])};
}

// identity of a secondary born from `parent` at `step` (splitmix64 finaliser)
__host__ __device__ __forceinline__ uint64_t child_id(uint64_t parent, int64_t step) {
  uint64_t z = parent + 0x9E3779B97F4A7C15ull * (uint64_t)(step + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// --------------------------------------------------------------- gather
// EM4.cu:41-122: staggered bilinear gather of Er (n_r x (n_z+1)), Ez
// ((n_r+1) x n_z), Hphi (n_r x n_z) at (r0, z0) with the reference's
// one-sided edge cases.  The row (column) index is clamped at z0 = Lp
// (r0 = Rp) exactly, where the reference reads past the array with weight 0.
// ldE, ldZ, ldH: row strides (elements) of Er, Ez and H.
template <typename T>
__device__ __forceinline__ void gather3s(const T *__restrict__ Er, const T *__restrict__ Ez,
                                         const T *__restrict__ H, int nr, int nz, int64_t ldE,
                                         int64_t ldZ, int64_t ldH, double dr, double dz, double r0,
                                         double z0, double &E_r, double &E_z, double &Hp) {
  int ar, az;
  int64_t a1, a2, a3, a4;
  ar = (int)floor(r0 / dr - 0.5);
  az = (int)floor(z0 / dz);
  if (az > nz - 1) az = nz - 1;
  a1 = ar + az * ldE; a2 = (ar + 1) + az * ldE;
  a3 = ar + (az + 1) * ldE; a4 = (ar + 1) + (az + 1) * ldE;
  if (ar < 0) E_r = ((double)Er[a2] * (az * dz + dz - z0) + (double)Er[a4] * (z0 - az * dz)) / dz;
  else if (ar >= nr - 1) E_r = ((double)Er[a1] * (az * dz + dz - z0) + (double)Er[a3] * (z0 - az * dz)) / dz;
  else
    E_r = ((double)Er[a1] * ((ar + 1.5) * dr - r0) * ((az + 1) * dz - z0) +
           (double)Er[a2] * (r0 - (ar + 0.5) * dr) * ((az + 1) * dz - z0) +
           (double)Er[a3] * ((ar + 1.5) * dr - r0) * (z0 - az * dz) +
           (double)Er[a4] * (r0 - (ar + 0.5) * dr) * (z0 - az * dz)) / (dr * dz);
  ar = (int)floor(r0 / dr);
  az = (int)floor(z0 / dz - 0.5);
  if (ar > nr - 1) ar = nr - 1;
  a1 = ar + az * ldZ; a2 = (ar + 1) + az * ldZ;
  a3 = ar + (az + 1) * ldZ; a4 = (ar + 1) + (az + 1) * ldZ;
  if (az < 0) E_z = ((double)Ez[a3] * (ar * dr + dr - r0) + (double)Ez[a4] * (r0 - ar * dr)) / dr;
  else if (az >= nz - 1) E_z = ((double)Ez[a1] * (ar * dr + dr - r0) + (double)Ez[a2] * (r0 - ar * dr)) / dr;
  else
    E_z = ((double)Ez[a1] * ((ar + 1) * dr - r0) * ((az + 1.5) * dz - z0) +
           (double)Ez[a2] * (r0 - ar * dr) * ((az + 1.5) * dz - z0) +
           (double)Ez[a3] * ((ar + 1) * dr - r0) * (z0 - (az + 0.5) * dz) +
           (double)Ez[a4] * (r0 - ar * dr) * (z0 - (az + 0.5) * dz)) / (dr * dz);
  ar = (int)floor(r0 / dr - 0.5);
  az = (int)floor(z0 / dz - 0.5);
  a1 = ar + az * ldH; a2 = (ar + 1) + az * ldH;
  a3 = ar + (az + 1) * ldH; a4 = (ar + 1) + (az + 1) * ldH;
  if (ar < 0) {
    if (az < 0) Hp = H[a4];
    else if (az >= nz - 1) Hp = H[a2];
    else Hp = ((double)H[a2] * ((az + 1.5) * dz - z0) + (double)H[a4] * (z0 - (az + 0.5) * dz)) / dz;
  } else if (ar >= nr - 1) {
    if (az < 0) Hp = H[a3];
    else if (az >= nz - 1) Hp = H[a1];
    else Hp = ((double)H[a1] * ((az + 1.5) * dz - z0) + (double)H[a3] * (z0 - (az + 0.5) * dz)) / dz;
  } else if (az < 0) {
    Hp = ((double)H[a3] * ((ar + 1.5) * dr - r0) + (double)H[a4] * (r0 - (ar + 0.5) * dr)) / dr;
  } else if (az >= nz - 1) {
    Hp = ((double)H[a1] * ((ar + 1.5) * dr - r0) + (double)H[a2] * (r0 - (ar + 0.5) * dr)) / dr;
  } else {
    Hp = ((double)H[a1] * ((ar + 1.5) * dr - r0) * ((az + 1.5) * dz - z0) +
          (double)H[a2] * (r0 - (ar + 0.5) * dr) * ((az + 1.5) * dz - z0) +
          (double)H[a3] * ((ar + 1.5) * dr - r0) * (z0 - (az + 0.5) * dz) +
          (double)H[a4] * (r0 - (ar + 0.5) * dr) * (z0 - (az + 0.5) * dz)) / (dr * dz);
  }
}

// the reference's dense column-major grids (EM4.cu:41-122)
template <typename T>
__device__ __forceinline__ void gather3(const T *__restrict__ Er, const T *__restrict__ Ez,
                                        const T *__restrict__ H, int nr, int nz, double dr,
                                        double dz, double r0, double z0, double &E_r,
                                        double &E_z, double &Hp) {
  gather3s<T>(Er, Ez, H, nr, nz, nr, nr + 1, nr, dr, dz, r0, z0, E_r, E_z, Hp);
}

// ------------------------------------------------------ deposit weights
// EM7.cu:56-162: the four cell-centred nodes around (r0, z0) and their
// bilinear weights, one-sided at the grid edges.  Returns ar (column of a1).
// ld: row stride (elements) of the current grid the indices a[] address.
__device__ __forceinline__ int em7_weights_ld(double r0, double z0, int nr, int nz, int64_t ld,
                                              double dr, double dz, int64_t a[4], double b[4]) {
  const int ar = (int)floor(r0 / dr - 0.5);
  const int az = (int)floor(z0 / dz - 0.5);
  a[0] = a[1] = a[2] = a[3] = 0;
  b[0] = b[1] = b[2] = b[3] = 0;
  if (ar < 0) {
    if (az < 0) { a[3] = (ar + 1) + (int64_t)(az + 1) * ld; b[3] = 1; }
    else if (az >= nz - 1) { a[1] = (ar + 1) + (int64_t)az * ld; b[1] = 1; }
    else {
      a[1] = (ar + 1) + (int64_t)az * ld; a[3] = (ar + 1) + (int64_t)(az + 1) * ld;
      b[1] = ((az + 1.5) * dz - z0) / (dz);
      b[3] = (z0 - (az + 0.5) * dz) / (dz);
    }
  } else if (ar >= nr - 1) {
    if (az < 0) { a[2] = ar + (int64_t)(az + 1) * ld; b[2] = 1; }
    else if (az >= nz - 1) { a[0] = ar + (int64_t)az * ld; b[0] = 1; }
    else {
      a[0] = ar + (int64_t)az * ld; a[2] = ar + (int64_t)(az + 1) * ld;
      b[0] = ((az + 1.5) * dz - z0) / (dz);
      b[2] = (z0 - (az + 0.5) * dz) / (dz);
    }
  } else {
    if (az < 0) {
      a[2] = ar + (int64_t)(az + 1) * ld; a[3] = (ar + 1) + (int64_t)(az + 1) * ld;
      b[2] = ((ar + 1.5) * dr - r0) / (dr);
      b[3] = (r0 - (ar + 0.5) * dr) / (dr);
    } else if (az >= nz - 1) {
      a[0] = ar + (int64_t)az * ld; a[1] = (ar + 1) + (int64_t)az * ld;
      b[0] = ((ar + 1.5) * dr - r0) / (dr);
      b[1] = (r0 - (ar + 0.5) * dr) / (dr);
    } else {
      a[0] = ar + (int64_t)az * ld; a[1] = (ar + 1) + (int64_t)az * ld;
      a[2] = ar + (int64_t)(az + 1) * ld; a[3] = (ar + 1) + (int64_t)(az + 1) * ld;
      b[0] = ((ar + 1.5) * dr - r0) * ((az + 1.5) * dz - z0) / (dr * dz);
      b[1] = (r0 - (ar + 0.5) * dr) * ((az + 1.5) * dz - z0) / (dr * dz);
      b[2] = ((ar + 1.5) * dr - r0) * (z0 - (az + 0.5) * dz) / (dr * dz);
      b[3] = (r0 - (ar + 0.5) * dr) * (z0 - (az + 0.5) * dz) / (dr * dz);
    }
  }
  return ar;
}

// the reference's dense n_r x n_z grid (EM7.cu:56-162)
__device__ __forceinline__ int em7_weights(double r0, double z0, int nr, int nz, double dr,
                                           double dz, int64_t a[4], double b[4]) {
  return em7_weights_ld(r0, z0, nr, nz, nr, dr, dz, a, b);
}

// fixed-point current: value * 2^S rounded to nearest, added with a 64-bit
// integer atomic (associative, so the grid is bit-identical run to run)
__device__ __forceinline__ void fx_add(unsigned long long *J, int64_t idx, double v, double scale) {
  const long long q = __double2ll_rn(v * scale);
  if (q != 0) atomicAdd(J + idx, (unsigned long long)q);
}

// shell volume of node column i (EM7.cu:175-176)
__host__ __device__ __forceinline__ double shell_volume(int i, double dr, double dz, double PHIp) {
  return PHIp / 2 * ((((i + 1) * dr) * ((i + 1) * dr) - (i * dr) * (i * dr)) * dz);
}

// ----------------------------------------------------------- half drift
// EM2.cu:26-57 / EM4.cu:146-177 in Cartesian form: drift by v dt/2, (r, phi),
// delete beyond Rp, wedge wrap that rotates the velocity-like vector w, and
// specular reflection at z = 0, Lp.  Corrected mode uses atan2 and skips the
// wrap for a full ring (PHIp >= 2 pi).
__device__ __forceinline__ void halfdrift_cart(double &x, double &y, double &z, double &wx,
                                               double &wy, double &wz, double vx, double vy,
                                               double vz, double &r_o, double &phi_o, int &del,
                                               double Rp, double Lp, double PHIp, double dt,
                                               unsigned flags) {
  double X = x + 0.5 * vx * dt;
  double Y = y + 0.5 * vy * dt;
  double Z = z + 0.5 * vz * dt;
  const double r = sqrt(X * X + Y * Y);
  double phi = (flags & GASATT_Q_ATAN_PHI) ? atan(Y / X) : atan2(Y, X);
  if (r > Rp) del = 1;
  const bool wrap = (flags & GASATT_Q_ATAN_PHI) || PHIp < 2 * GASATT_PI - 1e-12;
  if (wrap) {
    const double cp = cos(PHIp), sp = sin(PHIp);
    double w1;
    // bounded: a wrap count above 2^20 means phi is not finite-sized
    for (int it = 0; phi < 0 && it < (1 << 20); ++it) {
      phi = phi + PHIp;
      w1 = wx * cp - wy * sp;
      wy = wx * sp + wy * cp;
      wx = w1;
    }
    for (int it = 0; phi > PHIp && it < (1 << 20); ++it) {
      phi = phi - PHIp;
      w1 = wx * cp + wy * sp;
      wy = -wx * sp + wy * cp;
      wx = w1;
    }
  }
  X = r * cos(phi);
  Y = r * sin(phi);
  if (Z > Lp) { Z = 2 * Lp - Z; wz = -wz; }
  if (Z < 0) { Z = -Z; wz = -wz; }
  x = X; y = Y; z = Z;
  r_o = r; phi_o = phi;
}

// ------------------------------------------------------------- rotation
// electron_transport.cu:124-137 (rotate.m): turn (vx,vy,vz) by polar angle th
// and azimuth ph about itself.  ref_form selects the reference's perpendicular
// speed^2 expression v*v - vz*vz; otherwise vx*vx + vy*vy.
__device__ __forceinline__ void rotate_v(double &vx, double &vy, double &vz, double th,
                                         double ph, bool ref_form) {
  const double v = sqrt(vx * vx + vy * vy + vz * vz);
  const double p2 = ref_form ? v * v - vz * vz : vx * vx + vy * vy;
  double x0, y0, z0;
  if (p2 > 0.0001) {
    const double s = sqrt(p2);
    x0 = vx * cos(th) + sin(th) / s * (vx * vz * cos(ph) - v * vy * sin(ph));
    y0 = vy * cos(th) + sin(th) / s * (vy * vz * cos(ph) + v * vx * sin(ph));
    z0 = vz * cos(th) - s * sin(th) * cos(ph);
  } else {
    x0 = v * sin(th) * cos(ph);
    y0 = v * sin(th) * sin(ph);
    z0 = v * cos(th);
  }
  vx = x0; vy = y0; vz = z0;
}

// relativistic Boris push of u = gamma v (corrected kick)
__device__ __forceinline__ void boris(double &ux, double &uy, double &uz, double Ex, double Ey,
                                      double Ez, double Bx, double By, double Bz, double qm_dt2,
                                      double c) {
  const double umx = ux + qm_dt2 * Ex, umy = uy + qm_dt2 * Ey, umz = uz + qm_dt2 * Ez;
  const double gm = sqrt(1 + (umx * umx + umy * umy + umz * umz) / (c * c));
  const double f = qm_dt2 / gm;
  const double tx = f * Bx, ty = f * By, tz = f * Bz;
  const double t2 = tx * tx + ty * ty + tz * tz;
  const double upx = umx + (umy * tz - umz * ty);
  const double upy = umy + (umz * tx - umx * tz);
  const double upz = umz + (umx * ty - umy * tx);
  const double s = 2 / (1 + t2);
  const double sx = s * tx, sy = s * ty, sz = s * tz;
  const double wx = umx + (upy * sz - upz * sy);
  const double wy = umy + (upz * sx - upx * sz);
  const double wz = umz + (upx * sy - upy * sx);
  ux = wx + qm_dt2 * Ex; uy = wy + qm_dt2 * Ey; uz = wz + qm_dt2 * Ez;
}

}  // namespace gasatt
