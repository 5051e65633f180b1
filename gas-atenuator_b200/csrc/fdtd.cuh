// fdtd.cuh - axisymmetric Yee update (EM3_1.cu, EM3.cu) on the reference's
// staggering: Er n_r x (n_z+1) at ((i+1/2)dr, j dz), Ez (n_r+1) x n_z at
// (i dr, (j+1/2)dz), Hphi and j n_r x n_z at cell centres.  Column-major
// (r fastest).  Both updates run in place: the E update reads only its own
// old E value plus H and j, and the Er end rows that the reference copies
// from the first interior row (EM3.cu:21-27) are written by the thread that
// owns that interior row, from the value it read before updating it.
#pragma once
#include "gasatt_device.cuh"

namespace gasatt {

struct FdtdCoef {
  double chr, chz;        // dt/(mu dr), dt/(mu dz) for the H update (EM3_1.cu:95)
  double dt_eps;          // dt/eps
  double dt_eps_dz;       // dt/(eps dz)
  double axis;            // 4 dt/(eps dr)
  double dr;
  double inv_scale;       // 2^-S of the fixed-point current
  double dz, PHIp;        // shell volumes for the current density
};

// EM3_1.cu:89-95
template <typename T>
__global__ void k_fdtd_h(T *__restrict__ H, const T *__restrict__ Er, const T *__restrict__ Ez,
                         int nr, int nz, double chr, double chz) {
  const int64_t n = (int64_t)nr * nz;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % nr), j = (int)(idx / nr);
    const int64_t ez = i + (int64_t)j * (nr + 1);
    H[idx] = (T)((double)H[idx] + (chr * ((double)Ez[ez + 1] - (double)Ez[ez]) -
                                   chz * ((double)Er[idx + nr] - (double)Er[idx])));
  }
}

// current density [A/m^2] at a cell-centred node from the fixed-point sum of
// q FN v w over the particles
__device__ __forceinline__ double jdens(const unsigned long long *J, int64_t idx, int i,
                                        const FdtdCoef &c) {
  return (double)(long long)J[idx] * c.inv_scale / shell_volume(i, c.dr, c.dz, c.PHIp);
}

// EM3.cu:121-149
template <typename T>
__global__ void k_fdtd_e(T *__restrict__ Er, T *__restrict__ Ez, const T *__restrict__ H,
                         const unsigned long long *__restrict__ Jr,
                         const unsigned long long *__restrict__ Jz, int nr, int nz, FdtdCoef c,
                         unsigned flags) {
  const int64_t n = (int64_t)(nr + 1) * (nz + 1);
  const bool endcopy = (flags & GASATT_Q_ER_END_COPY) != 0;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % (nr + 1)), j = (int)(idx / (nr + 1));
    const int64_t n_r = i + (int64_t)j * nr, n_z = i + (int64_t)j * (nr + 1);
    if (i < nr) {
      if (j >= 1 && j < nz) {
        const double old = (double)Er[n_r];
        const double ja = jdens(Jr, n_r - nr, i, c), jb = jdens(Jr, n_r, i, c);
        Er[n_r] = (T)(old - c.dt_eps * (ja + jb) / 2 -
                      c.dt_eps_dz * ((double)H[n_r] - (double)H[n_r - nr]));
        if (endcopy) {
          if (j == 1) Er[i] = (T)old;
          if (j == nz - 1) Er[i + (int64_t)nz * nr] = (T)old;
        }
      } else if (!endcopy) {
        Er[n_r] = (T)0;                      // conducting end wall
      }
    }
    if (j < nz) {
      if (i < 1) {
        const double jz0 = jdens(Jz, n_r, 0, c);
        const double jterm = (flags & GASATT_Q_EZ_AXIS_JSIGN) ? c.dt_eps * jz0 : -(c.dt_eps * jz0);
        Ez[n_z] = (T)((double)Ez[n_z] + jterm + c.axis * (double)H[n_r]);
      } else if (i < nr) {
        const double ri = (flags & GASATT_Q_EZ_RSHIFT) ? (i + 1) * c.dr : i * c.dr;
        const double ja = jdens(Jz, n_r - 1, i - 1, c), jb = jdens(Jz, n_r, i, c);
        Ez[n_z] = (T)((double)Ez[n_z] - c.dt_eps * (ja + jb) / 2 +
                      c.dt_eps * (1 / (2 * ri) + 1 / c.dr) * (double)H[n_r] +
                      c.dt_eps * (1 / (2 * ri) - 1 / c.dr) * (double)H[n_r - 1]);
      }
    }
  }
}

}  // namespace gasatt
