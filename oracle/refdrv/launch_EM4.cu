/* Driver for the reference EM4.cu (gather + kick + half drift). */
#include "refdrv.h"
#include REF_SRC
extern "C" int ref_EM4(double *x, double *y, double *z, double *vx, double *vy, double *vz,
                       double *r, double *phi, double *vr, double *Er, double *Ez, double *H,
                       double *q, double *m, double *E, int *del, int n, double Rp, double Lp,
                       double PHIp, int gridR, int gridZ, double mu, double c, double dr,
                       double dz, double dt) {
  double *d[15];
  double *h[15] = {x, y, z, vx, vy, vz, r, phi, vr, Er, Ez, H, q, m, E};
  size_t N = (size_t)n;
  size_t sz[15] = {N, N, N, N, N, N, N, N, N, (size_t)gridR * (gridZ + 1),
                   (size_t)(gridR + 1) * gridZ, (size_t)gridR * gridZ, N, N, N};
  int *dd;
  for (int i = 0; i < 15; ++i) RD_UP(d[i], h[i], sz[i]);
  RD_UP(dd, del, N);
  processMandelbrotElement<<<(n + 1023) / 1024 > 0 ? (n + 1023) / 1024 : 1, 1024>>>(
      d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7], d[8], d[9], d[10], d[11], d[12], d[13],
      d[14], dd, n, Rp, Lp, PHIp, gridR, gridZ, mu, c, dr, dz, dt);
  RD_CHECK(cudaGetLastError()); RD_CHECK(cudaDeviceSynchronize());
  for (int i = 0; i < 15; ++i) { RD_DOWN(h[i], d[i], sz[i]); cudaFree(d[i]); }
  RD_DOWN(del, dd, N); cudaFree(dd);
  return 0;
}
