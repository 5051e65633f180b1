/* Driver for the reference EM2.cu (half drift + wedge/z boundary). */
#include "refdrv.h"
#include REF_SRC
extern "C" int ref_EM2(double *x, double *y, double *z, double *vx, double *vy, double *vz,
                       double *r, double *phi, double *vr, int *del, int n, double Rp,
                       double Lp, double PHIp, double dr, double dz, double dt) {
  double *d[9]; double *h[9] = {x, y, z, vx, vy, vz, r, phi, vr}; int *dd;
  for (int i = 0; i < 9; ++i) RD_UP(d[i], h[i], (size_t)n);
  RD_UP(dd, del, (size_t)n);
  processMandelbrotElement<<<(n + 1023) / 1024 > 0 ? (n + 1023) / 1024 : 1, 1024>>>(
      d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7], d[8], dd, n, Rp, Lp, PHIp, dr, dz, dt);
  RD_CHECK(cudaGetLastError()); RD_CHECK(cudaDeviceSynchronize());
  for (int i = 0; i < 9; ++i) { RD_DOWN(h[i], d[i], (size_t)n); cudaFree(d[i]); }
  RD_DOWN(del, dd, (size_t)n); cudaFree(dd);
  return 0;
}
