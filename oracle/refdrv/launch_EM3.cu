/* Driver for the reference EM3.cu (E update); launch shape as
 * electricmagneticfield6.m:86-87: n_r+1 threads, n_z+1 blocks.  Er0/Ez0 and
 * Er/Ez are separate buffers, as feval's copies make them. */
#include "refdrv.h"
#include REF_SRC
extern "C" int ref_EM3(double *Er0, double *Ez0, double *H0, double *Er, double *Ez,
                       double *jr, double *jz, int nr, int nz, double mu, double eps,
                       double dr, double dz, double dt) {
  if (nr + 1 > 1024) return 1;
  size_t ner = (size_t)nr * (nz + 1), nez = (size_t)(nr + 1) * nz, nh = (size_t)nr * nz;
  double *a, *b, *c, *d, *e, *f, *g;
  RD_UP(a, Er0, ner); RD_UP(b, Ez0, nez); RD_UP(c, H0, nh); RD_UP(d, Er, ner);
  RD_UP(e, Ez, nez); RD_UP(f, jr, nh); RD_UP(g, jz, nh);
  processMandelbrotElement<<<nz + 1, nr + 1>>>(a, b, c, d, e, f, g, mu, eps, dr, dz, dt);
  RD_CHECK(cudaGetLastError()); RD_CHECK(cudaDeviceSynchronize());
  RD_DOWN(Er, d, ner); RD_DOWN(Ez, e, nez);
  cudaFree(a); cudaFree(b); cudaFree(c); cudaFree(d); cudaFree(e); cudaFree(f); cudaFree(g);
  return 0;
}
