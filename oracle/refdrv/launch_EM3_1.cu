/* Driver for the reference EM3_1.cu (H update); launch shape as
 * electricmagneticfield6.m:92-93: n_r threads, n_z blocks. */
#include "refdrv.h"
#include REF_SRC
extern "C" int ref_EM3_1(double *Er, double *Ez, double *H, int nr, int nz, double mu,
                         double dr, double dz, double dt) {
  if (nr > 1024) return 1;
  double *dEr, *dEz, *dH;
  RD_UP(dEr, Er, (size_t)nr * (nz + 1)); RD_UP(dEz, Ez, (size_t)(nr + 1) * nz);
  RD_UP(dH, H, (size_t)nr * nz);
  processMandelbrotElement<<<nz, nr>>>(dEr, dEz, dH, mu, dr, dz, dt);
  RD_CHECK(cudaGetLastError()); RD_CHECK(cudaDeviceSynchronize());
  RD_DOWN(H, dH, (size_t)nr * nz);
  cudaFree(dEr); cudaFree(dEz); cudaFree(dH);
  return 0;
}
