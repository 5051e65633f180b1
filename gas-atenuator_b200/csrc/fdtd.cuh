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

namespace gasatt {

// Packed gather quads of the FP32 form: for each interpolation cell of a
// field, its four (edge-clamped) corner values as one float4, so the particle
// pass reads one 16-byte vector per field instead of four scalars and needs no
// clamping.  Indices (ar, az: the half-cell shifted column and row of a
// particle, from -1; ir, iz: its cell):
//   Er: (ar + 1) + iz (n_r + 1)        corners (max(ar,0) | min(ar+1,n_r-1)) x (iz | iz+1)
//   Ez: ir + (az + 1) n_r              corners (ir | ir+1) x (max(az,0) | min(az+1,n_z-1))
//   H:  (ar + 1) + (az + 1) (n_r + 1)  corners as Er's columns x Ez's rows
// in the order (c0,r0), (c1,r0), (c0,r1), (c1,r1).
struct FieldQuads {
  float4 *er, *ez, *h;
};

// The quad slots that read field value (i, j) along one axis: a "shifted"
// axis (quads 0..n, corners max(q-1,0) and min(q,n-1)) or a "plain" one
// (quads 0..n-1, corners q and q+1).  Four fixed (quad, corner) slots, m the
// mask of those that apply (fixed slots keep the arrays in registers).
struct QuadAxis {
  int q[4], d[4];
  unsigned m;
};
__device__ __forceinline__ QuadAxis quad_axis_shifted(int i, int n) {
  QuadAxis a;
  a.q[0] = i + 1; a.d[0] = 0;
  a.q[1] = i;     a.d[1] = 1;
  a.q[2] = 0;     a.d[2] = 0;        // the clamped low edge reads value 0 twice
  a.q[3] = n;     a.d[3] = 1;        // the clamped high edge reads value n-1 twice
  a.m = 3u | (i == 0 ? 4u : 0u) | (i == n - 1 ? 8u : 0u);
  return a;
}
__device__ __forceinline__ QuadAxis quad_axis_plain(int i, int n) {
  QuadAxis a;
  a.q[0] = i;     a.d[0] = 0;
  a.q[1] = i - 1; a.d[1] = 1;
  a.q[2] = 0;     a.d[2] = 0;
  a.q[3] = 0;     a.d[3] = 0;
  a.m = (i < n ? 1u : 0u) | (i > 0 ? 2u : 0u);
  return a;
}
__device__ __forceinline__ void quad_put(float4 *Q, int ncq, const QuadAxis &cx,
                                         const QuadAxis &ry, float v) {
  float *f = reinterpret_cast<float *>(Q);
#pragma unroll
  for (int a = 0; a < 4; ++a) {
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      if (((cx.m >> a) & 1u) && ((ry.m >> b) & 1u))
        f[(((int64_t)cx.q[a] + (int64_t)ry.q[b] * ncq) << 2) + cx.d[a] + 2 * ry.d[b]] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// Fused field sub-cycle for the resident simulation: one launch advances the
// fields by one particle step, H(dt/4), [E(dt/2), H(dt/2)] x (2R - 1), E(dt/2),
// H(dt/4) (the reference's H(-dt/4) [H(dt/2) E(dt/2)] x 2R H(dt/4) with the
// first two H updates merged).  Each block loads a 32 x 32 patch = a tile of
// (32 - 4R - 1)^2 cells plus a halo of 2R cells on the low side and 2R + 1 on
// the high side (each H update needs E one cell up in r and z, each E update
// needs H one cell down) into shared memory, runs all sub-updates there, and
// writes its tile to the output fields (a second buffer: the patches of other
// blocks, which may run later, still read the old fields around this tile).
// A warp covers one 32-cell row of the patch.  The
// current it reads (Jr, Jz, fixed point) was deposited by the previous
// particle pass; the block clears its tile of the other buffer (Jr_next,
// Jz_next) for the next pass.  Storage in T; the patch stays in shared
// memory in double for the whole sub-cycle, so the FP32 form rounds its
// fields to float once per step and converts once each way.
constexpr int kFdtdPatch = 32;
constexpr int kFdtdRows = 16;                          // blockDim = (32, kFdtdRows)

__host__ __device__ inline int fdtd_tile(int R) { return kFdtdPatch - 4 * R - 1; }

// A second fixed-point current added to the first (the held ion current of
// the resident simulation), in units of rel x the first one's; Jr null: none.
struct ExtraCurrent {
  const unsigned long long *Jr, *Jz;
  double rel;
};

template <typename T>
__device__ __forceinline__ void fdtd_tiled(const T *__restrict__ Er, const T *__restrict__ Ez,
                                           const T *__restrict__ H, T *__restrict__ Er_out,
                                           T *__restrict__ Ez_out, T *__restrict__ H_out,
                                           const unsigned long long *__restrict__ Jr,
                                           const unsigned long long *__restrict__ Jz,
                                           unsigned long long *__restrict__ Jr_next,
                                           unsigned long long *__restrict__ Jz_next, int nr,
                                           int nz, int ldf, int ldj, const FdtdCoef &c,
                                           const double *__restrict__ invV, double mu, double dt,
                                           int R, unsigned flags, ExtraCurrent xj, FieldQuads q) {
  constexpr int TW = kFdtdPatch;
  __shared__ double sEr[TW * TW], sEz[TW * TW], sH[TW * TW], sJr[TW * TW], sJz[TW * TW];
  const int tile = fdtd_tile(R), hl = 2 * R, hh = 2 * R + 1;
  const int i0 = blockIdx.x * tile, j0 = blockIdx.y * tile;
  const int I0 = max(i0 - hl, 0), J0 = max(j0 - hl, 0);
  const int I1 = min(i0 + tile + hh, nr + 1), J1 = min(j0 + tile + hh, nz + 1);
  const int W = I1 - I0, Hn = J1 - J0;
  const int li = threadIdx.x, i = I0 + li;
  const bool col = li < W;
  for (int lj = threadIdx.y; lj < Hn; lj += kFdtdRows) {
    const int j = J0 + lj, s = li + lj * TW;
    if (!col) continue;
    if (i < nr && j <= nz) sEr[s] = (double)Er[i + (int64_t)j * ldf];
    if (i <= nr && j < nz) sEz[s] = (double)Ez[i + (int64_t)j * ldf];
    if (i < nr && j < nz) {
      const int64_t g = i + (int64_t)j * ldj;
      sH[s] = (double)H[i + (int64_t)j * ldf];
      if (xj.Jr) {
        sJr[s] = ((double)(long long)Jr[g] + (double)(long long)xj.Jr[g] * xj.rel) * invV[i];
        sJz[s] = ((double)(long long)Jz[g] + (double)(long long)xj.Jz[g] * xj.rel) * invV[i];
      } else {
        sJr[s] = (double)(long long)Jr[g] * invV[i];
        sJz[s] = (double)(long long)Jz[g] * invV[i];
      }
    }
  }
  __syncthreads();
  const bool endcopy = (flags & GASATT_Q_ER_END_COPY) != 0;
  const double dt_eps = c.dt_eps, dt_eps_dz = c.dt_eps_dz, axis = c.axis, inv_dr = 1 / c.dr;
  const double ri = ((flags & GASATT_Q_EZ_RSHIFT) ? (i + 1) : i) * c.dr;
  const double ezp = i > 0 ? dt_eps * (1 / (2 * ri) + inv_dr) : 0.0;   // coefficient of H(i)
  const double ezm = i > 0 ? dt_eps * (1 / (2 * ri) - inv_dr) : 0.0;   // coefficient of H(i-1)
  const int nsub = 4 * R + 1;
  for (int sub = 0; sub < nsub; ++sub) {
    if ((sub & 1) == 0) {                              // H update
      const double h = (sub == 0 || sub == nsub - 1) ? dt / 4 : dt / 2;
      const double chr = h / (mu * c.dr), chz = h / (mu * c.dz);
      if (col && i < nr && i + 1 < I1) {
        for (int lj = threadIdx.y; lj < Hn; lj += kFdtdRows) {
          const int j = J0 + lj, s = li + lj * TW;
          if (j < nz && j + 1 < J1)
            sH[s] = sH[s] + (chr * (sEz[s + 1] - sEz[s]) - chz * (sEr[s + TW] - sEr[s]));
        }
      }
    } else if (col) {                                  // E update (dt/2)
      for (int lj = threadIdx.y; lj < Hn; lj += kFdtdRows) {
        const int j = J0 + lj, s = li + lj * TW;
        if (i < nr) {
          if (j >= 1 && j < nz) {
            if (j - 1 >= J0) {
              const double old = sEr[s];
              sEr[s] = old - dt_eps * (sJr[s - TW] + sJr[s]) / 2 - dt_eps_dz * (sH[s] - sH[s - TW]);
              if (endcopy) {
                if (j == 1 && J0 == 0) sEr[s - TW] = old;
                if (j == nz - 1 && J1 == nz + 1) sEr[s + TW] = old;
              }
            }
          } else if (!endcopy && j <= nz) {
            sEr[s] = 0.0;
          }
        }
        if (j < nz) {
          if (i == 0) {
            const double jz0 = sJz[s];
            const double jterm = (flags & GASATT_Q_EZ_AXIS_JSIGN) ? dt_eps * jz0 : -(dt_eps * jz0);
            sEz[s] = sEz[s] + jterm + axis * sH[s];
          } else if (i < nr && i - 1 >= I0) {
            sEz[s] = sEz[s] - dt_eps * (sJz[s - 1] + sJz[s]) / 2 + ezp * sH[s] + ezm * sH[s - 1];
          }
        }
      }
    }
    __syncthreads();
  }
  const int ie = min(i0 + tile, nr + 1), je = min(j0 + tile, nz + 1);
  if (i >= i0 && i < ie) {
    for (int j = J0 + threadIdx.y; j < je; j += kFdtdRows) {
      if (j < j0) continue;
      const int s = li + (j - J0) * TW;
      if (i < nr && j <= nz) {
        const T v = (T)sEr[s];
        Er_out[i + (int64_t)j * ldf] = v;
        if (q.er) quad_put(q.er, nr + 1, quad_axis_shifted(i, nr), quad_axis_plain(j, nz), (float)v);
      }
      if (i <= nr && j < nz) {
        const T v = (T)sEz[s];
        Ez_out[i + (int64_t)j * ldf] = v;
        if (q.ez) quad_put(q.ez, nr, quad_axis_plain(i, nr), quad_axis_shifted(j, nz), (float)v);
      }
      if (i < nr && j < nz) {
        const int64_t g = i + (int64_t)j * ldj;
        const T v = (T)sH[s];
        H_out[i + (int64_t)j * ldf] = v;
        if (q.h) quad_put(q.h, nr + 1, quad_axis_shifted(i, nr), quad_axis_shifted(j, nz), (float)v);
        Jr_next[g] = 0;
        Jz_next[g] = 0;
      }
    }
  }
}

}  // namespace gasatt
