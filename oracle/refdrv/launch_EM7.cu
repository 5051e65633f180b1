/* Driver for the reference EM7.cu (bilinear current deposition). */
#include "refdrv.h"
#include REF_SRC
extern "C" int ref_EM7(double *r, double *z, double *q, double *vr, double *vz, double *jr,
                       double *jz, int *del, int n, int gridR, int gridZ, double dr, double dz,
                       double FN, double PHIp) {
  double *d[7]; double *h[7] = {r, z, q, vr, vz, jr, jz}; int *dd;
  size_t sz[7] = {(size_t)n, (size_t)n, (size_t)n, (size_t)n, (size_t)n,
                  (size_t)gridR * gridZ, (size_t)gridR * gridZ};
  for (int i = 0; i < 7; ++i) RD_UP(d[i], h[i], sz[i]);
  RD_UP(dd, del, (size_t)n);
  processMandelbrotElement<<<(n + 1023) / 1024 > 0 ? (n + 1023) / 1024 : 1, 1024>>>(
      d[0], d[1], d[2], d[3], d[4], d[5], d[6], dd, n, gridR, gridZ, dr, dz, FN, PHIp);
  RD_CHECK(cudaGetLastError()); RD_CHECK(cudaDeviceSynchronize());
  RD_DOWN(jr, d[5], sz[5]); RD_DOWN(jz, d[6], sz[6]);
  for (int i = 0; i < 7; ++i) cudaFree(d[i]);
  cudaFree(dd);
  return 0;
}
