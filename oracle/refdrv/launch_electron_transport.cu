/* Driver for the reference electron_transport.cu (MCC) with injected draws
 * (rng_shim.h is force-included ahead of the reference source). */
#include "refdrv.h"
#include REF_SRC
extern "C" int ref_electron_transport(
    double *x, double *y, double *z, double *vx, double *vy, double *vz, double *sig_el,
    double *sig_ion, double *sig_exc, double *energy, double *xI, double *yI, double *V,
    int ne, double *density, double *temperature, int ncell, double *dphi, int rmax,
    double *kExc, double *Aexc, double *omExc, double *vExc, double *gaExc, int lenExc,
    unsigned char *sec, double *svx, double *svy, double *svz, double *sample, double *ivx,
    double *ivy, double *ivz, int *sum_cell0, int cellnumxy, double dr, double dz, double dt,
    int n, const double *draws) {
  size_t N = (size_t)n;
  double *dp[10]; double *hp[10] = {x, y, z, vx, vy, vz, sig_el, sig_ion, sig_exc, energy};
  for (int i = 0; i < 10; ++i) RD_UP(dp[i], hp[i], N);
  double *dxI, *dyI, *dV, *dden, *dtem, *ddphi, *de[5]; double *he[5] = {kExc, Aexc, omExc, vExc, gaExc};
  RD_UP(dxI, xI, (size_t)ne); RD_UP(dyI, yI, (size_t)ne); RD_UP(dV, V, (size_t)ne * 181);
  RD_UP(dden, density, (size_t)ncell); RD_UP(dtem, temperature, (size_t)ncell);
  RD_UP(ddphi, dphi, (size_t)rmax);
  for (int i = 0; i < 5; ++i) RD_UP(de[i], he[i], (size_t)lenExc);
  bool *dsec; RD_CHECK(cudaMalloc((void **)&dsec, N ? N : 1)); RD_CHECK(cudaMemcpy(dsec, sec, N, cudaMemcpyHostToDevice));
  double *dq[7]; double *hq[7] = {svx, svy, svz, sample, ivx, ivy, ivz};
  for (int i = 0; i < 7; ++i) RD_UP(dq[i], hq[i], N);
  int *dsc; RD_UP(dsc, sum_cell0, (size_t)rmax + 1);
  double *ddraw; RD_UP(ddraw, draws, N * 8);
  RD_CHECK(cudaMemcpyToSymbol(g_shim_draws, &ddraw, sizeof(ddraw)));
  processMandelbrotElement<<<(n + 255) / 256 > 0 ? (n + 255) / 256 : 1, 256>>>(
      dp[0], dp[1], dp[2], dp[3], dp[4], dp[5], dp[6], dp[7], dp[8], dp[9], dxI, dyI, dV, dden,
      dtem, ddphi, de[0], de[1], de[2], de[3], de[4], dsec, dq[0], dq[1], dq[2], dq[3], dq[4],
      dq[5], dq[6], dsc, lenExc, cellnumxy, dr, dz, dt, n);
  RD_CHECK(cudaGetLastError()); RD_CHECK(cudaDeviceSynchronize());
  for (int i = 3; i < 6; ++i) RD_DOWN(hp[i], dp[i], N);
  RD_CHECK(cudaMemcpy(sec, dsec, N, cudaMemcpyDeviceToHost));
  for (int i = 0; i < 7; ++i) RD_DOWN(hq[i], dq[i], N);
  for (int i = 0; i < 10; ++i) cudaFree(dp[i]);
  for (int i = 0; i < 7; ++i) cudaFree(dq[i]);
  for (int i = 0; i < 5; ++i) cudaFree(de[i]);
  cudaFree(dxI); cudaFree(dyI); cudaFree(dV); cudaFree(dden); cudaFree(dtem); cudaFree(ddphi);
  cudaFree(dsec); cudaFree(dsc); cudaFree(ddraw);
  return 0;
}
