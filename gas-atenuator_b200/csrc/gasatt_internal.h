// gasatt_internal.h - host-side context, error handling and table builders.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>
#include "../../include/gasatt.h"

struct gasatt_ctx {
  int device = 0;
  uint64_t seed = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int64_t launches = 0;      // kernels launched by this context
  int64_t mcc_calls = 0;     // gasatt_electron_collision calls (Philox counter)
  // reusable device scratch (grown on demand)
  void *scratch = nullptr;
  size_t scratch_bytes = 0;
  void *pinned = nullptr;    // small pinned host buffer for counters
};

namespace gasatt {

int fail(gasatt_ctx *ctx, int code, const std::string &msg);
int cuda_fail(gasatt_ctx *ctx, cudaError_t e, const char *what);
// device scratch of at least `bytes`, owned by the context
int scratch(gasatt_ctx *ctx, size_t bytes, void **ptr);

#define GASATT_CUDA(ctx, call)                                        \
  do {                                                                \
    cudaError_t e__ = (call);                                         \
    if (e__ != cudaSuccess) return gasatt::cuda_fail((ctx), e__, #call); \
  } while (0)
#define GASATT_LAUNCHED(ctx)                                          \
  do {                                                                \
    (ctx)->launches++;                                                \
    cudaError_t e__ = cudaGetLastError();                             \
    if (e__ != cudaSuccess) return gasatt::cuda_fail((ctx), e__, "kernel launch"); \
  } while (0)

inline unsigned grid_for(int64_t n, int block, unsigned cap = 148u * 32u) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

// ---- tables (host) ----
// electron_collision.m:12-33: combined elastic tables, ne energies.
struct ElasticTables {
  int ne = 0;
  std::vector<double> xInterp, yInterp, V;   // V: 181 x ne, column per energy
};
int build_elastic_tables(const gasatt_tables *t, ElasticTables &out, std::string &err);
int check_tables(const gasatt_tables *t, std::string &err);

// find_CS0.m on one energy (keV); flags: GASATT_Q_XS_NAN
void find_cs0_host(const gasatt_tables *t, double E_keV, double &se, double &si, double &sx,
                   unsigned flags);

// Resident-simulation tables: cross-sections on G log-spaced energies, the
// normalised elastic CDF per grid energy, and the FP64 null-collision bound.
struct SimTables {
  int G = 0;
  double lnEmin = 0, dlnE = 0;
  std::vector<double> sig_el, sig_ion, sig_exc, cdf;   // G, G, G, G*181
  std::vector<double> edep;                            // G: mean excitation loss [eV]
  double exc_kmin = 0;                                 // lowest excitation threshold [eV]
  double nu_max = 0;
  double sigv_max = 0;   // max over the table of sigma_tot(E) v(E) [m^3/s]
  int n_exc = 0;
  double exc[5][16] = {};   // k, A, omega, nu, gamma
};
int build_sim_tables(const gasatt_tables *t, int G, double emin_ev, double emax_ev, double n_gas,
                     double c, double me, double qe, SimTables &out, std::string &err);

}  // namespace gasatt
