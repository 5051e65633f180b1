// dropin.cu - CUDA drop-ins for the reference driver's MATLAB functions:
//   find_CS0, free_motion, particle_density, electricmagneticfield6
//   (EM2 + EM7 + EM3_1 + EM3 + EM4), electron_collision (electron_transport).
// Plain FP64 on the MATLAB column-major arrays; compiled with -fmad=false so
// the arithmetic follows the reference expression by expression.
#include <cub/device/device_scan.cuh>
#include <cmath>
#include <cstring>
#include <string>
#include "fdtd.cuh"
#include "gasatt_internal.h"

using namespace gasatt;

namespace {

constexpr int kBlock = 256;

// ------------------------------------------------------------- find_CS0
struct XsRaw {            // device copies of the raw find_CS0 tables
  const double *t_el; int n_el;
  const double *t_sel; int n_sel;
  const double *t_ion; int n_ion;
  const double *t_exc; int n_exc;
};

__device__ double d_interp1(const double *x, int sx, const double *y, int sy, int n, double xq) {
  if (!(xq >= x[0] && xq <= x[(int64_t)(n - 1) * sx])) return nan("");
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (x[(int64_t)mid * sx] <= xq) lo = mid; else hi = mid;
  }
  const double x0 = x[(int64_t)lo * sx], x1 = x[(int64_t)hi * sx];
  const double y0 = y[(int64_t)lo * sy], y1 = y[(int64_t)hi * sy];
  return y0 + (xq - x0) * (y1 - y0) / (x1 - x0);
}

__device__ double d_loglog(const double *x, int sx, const double *y, int sy, int n, double xq) {
  const double x0 = x[(int64_t)(n - 2) * sx], x1 = x[(int64_t)(n - 1) * sx];
  const double y0 = y[(int64_t)(n - 2) * sy], y1 = y[(int64_t)(n - 1) * sy];
  const double s = log(y1 / y0) / log(x1 / x0);
  return y1 * pow(xq / x1, s);
}

// find_CS0.m:100-146 on one energy E [keV]
__global__ void k_find_cs0(XsRaw t, const double *__restrict__ E, int64_t n, double *se,
                           double *si, double *sx, unsigned flags) {
  const bool faithful = (flags & GASATT_Q_XS_NAN) != 0;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const double e = E[p];
    double sel = 0.0;
    if (e >= 0.05) {
      sel = d_interp1(&t.t_el[0], 2, &t.t_el[1], 2, t.n_el, e);
      if (!faithful && e > t.t_el[2 * (t.n_el - 1)]) sel = d_loglog(&t.t_el[0], 2, &t.t_el[1], 2, t.n_el, e);
      sel = sel * GASATT_A0SQ * 2;
    } else if (e < 0.05) {
      double Ev = e * 1000;
      if (!faithful && Ev < t.t_sel[0]) Ev = t.t_sel[0];
      sel = d_interp1(&t.t_sel[0], 1, &t.t_sel[t.n_sel], 1, t.n_sel, Ev) * 1e-20;
    }
    se[p] = sel;
    const double T = e * 1000;
    double sion;
    if (!faithful && T <= t.t_ion[0]) sion = 0.0;
    else if (!faithful && T > t.t_ion[t.n_ion - 1])
      sion = d_loglog(&t.t_ion[0], 1, &t.t_ion[t.n_ion], 1, t.n_ion, T) * 1e-20;
    else sion = d_interp1(&t.t_ion[0], 1, &t.t_ion[t.n_ion], 1, t.n_ion, T) * 1e-20;
    si[p] = sion;
    double s = 0.0;
    for (int i = 0; i < t.n_exc; ++i) {
      const double k = t.t_exc[i], A = t.t_exc[t.n_exc + i], om = t.t_exc[2 * t.n_exc + i];
      const double nu = t.t_exc[3 * t.n_exc + i], ga = t.t_exc[4 * t.n_exc + i];
      if (!faithful && !(T > k)) continue;
      const double a = GASATT_CS_Q0 * A / (k * k);
      const double b = pow(k / T, om);
      const double c = pow(1 - pow(k / T, ga), nu);
      s = s + a * b * c;
    }
    sx[p] = s * 1e-4;
  }
}

// ---------------------------------------------------------- free_motion
__global__ void k_free_motion(const double *vx, const double *vy, const double *vz,
                              const double *x, const double *y, const double *z, int64_t n,
                              double dt, double *xn, double *yn, double *zn, double *rn,
                              double *phin) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double X = x[i] + vx[i] * dt, Y = y[i] + vy[i] * dt, Z = z[i] + vz[i] * dt;
    xn[i] = X; yn[i] = Y; zn[i] = Z;
    rn[i] = sqrt(X * X + Y * Y);
    phin[i] = atan2(Y, X);
  }
}

// ---------------------------------------------------------------- REBOND
// REBOND.m:6-66: an azimuth below 0 is raised by PHIp, with (v1, v2) turned
// by +PHIp, until it is not; the wrapped particle's x, y are rebuilt from r
// and the new azimuth; the same downwards above PHIp; then specular
// reflection at z = Lp and at z = 0.  Each wrap or reflection is one boundary
// event (count[0]).  The reference loops until every azimuth is inside; here a
// particle stops after kRebondMaxWraps wraps and raises count[1] (the call
// then fails) instead of looping without end on a wild azimuth.
constexpr int kRebondMaxWraps = 4096;

__global__ void k_rebond(double *pos, int64_t ldp, const double *r, const double *phi,
                         double *vel, int64_t ldv, int64_t n, double Lp, double PHIp, double cP,
                         double sP, unsigned long long *count) {
  unsigned long long ev = 0, bad = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double ph = phi[i], v1 = vel[i], v2 = vel[ldv + i];
    int k = 0;
    if (ph < 0) {
      while (ph < 0 && k < kRebondMaxWraps) {
        ph = ph + PHIp;
        const double w = v1 * cP - v2 * sP;
        v2 = v1 * sP + v2 * cP;
        v1 = w;
        ++k;
      }
      pos[i] = r[i] * cos(ph);
      pos[ldp + i] = r[i] * sin(ph);
    }
    if (ph > PHIp) {
      while (ph > PHIp && k < kRebondMaxWraps) {
        ph = ph - PHIp;
        const double w = v1 * cP + v2 * sP;
        v2 = -v1 * sP + v2 * cP;
        v1 = w;
        ++k;
      }
      pos[i] = r[i] * cos(ph);
      pos[ldp + i] = r[i] * sin(ph);
    }
    if (ph < 0 || ph > PHIp) bad++;
    vel[i] = v1;
    vel[ldv + i] = v2;
    double z = pos[2 * ldp + i], vz = vel[2 * ldv + i];
    if (z > Lp) { z = 2 * Lp - z; vz = -vz; ++k; }
    if (z < 0) { z = -z; vz = -vz; ++k; }
    pos[2 * ldp + i] = z;
    vel[2 * ldv + i] = vz;
    ev += (unsigned long long)k;
  }
  for (int o = 16; o; o >>= 1) {
    ev += __shfl_down_sync(0xFFFFFFFFu, ev, o);
    bad += __shfl_down_sync(0xFFFFFFFFu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (ev) atomicAdd(count, ev);
    if (bad) atomicAdd(count + 1, bad);
  }
}

// ------------------------------------------------------ particle_density
// particle_density.m:24-28: 1-based cell index via MATLAB round(x/d + 0.5)
__global__ void k_density_count(double dr, double dz, const double *dphi, int rmax,
                                const double *r, const double *phi, const double *z, int64_t n,
                                int cellnumxy, const double *sum_cell, int64_t ncell,
                                unsigned long long *count) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const double iz = round(z[p] / dz + 0.5), ir = round(r[p] / dr + 0.5);
    if (!(ir >= 1 && ir <= rmax)) continue;
    const double ip = round(phi[p] / dphi[(int)ir - 1] + 0.5);
    const double base = ((int)ir != 1) ? sum_cell[(int)ir - 2] : 0.0;
    const double idx = (iz - 1) * cellnumxy + base + ip;
    if (!(idx >= 1 && idx <= (double)ncell)) continue;
    atomicAdd(count + ((int64_t)idx - 1), 1ull);
  }
}

__global__ void k_density_finish(const unsigned long long *count, int64_t ncell, int cellnumxy,
                                 const double *VC, double FN, double *density) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncell;
       c += (int64_t)gridDim.x * blockDim.x)
    density[c] = FN * (double)count[c] / VC[c % cellnumxy];
}

// Per-cell counters of gasatt_particle_density_noalloc: a fixed array in the
// library's device image, so that call needs no device allocation.  In host
// code the name g_density_counts stands for a host-side shadow, not a device
// address; the device address comes from cudaGetSymbolAddress with the
// device current.
static __device__ __align__(256) unsigned long long
    g_density_counts[GASATT_DENSITY_NOALLOC_MAX_CELLS];

// Device address of g_density_counts on the current device, looked up on
// every call: a cached address would go stale when the device's primary
// context is reset (cudaDeviceReset, or MATLAB's reset(gpuDevice)) and the
// module is loaded again elsewhere.  Once the module is loaded the lookup is
// a table read.
int density_counts_on_device(gasatt_ctx *ctx, unsigned long long **out) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_density_counts);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGetSymbolAddress(g_density_counts)");
  *out = static_cast<unsigned long long *>(p);
  return GASATT_OK;
}

// -------------------------------------------- electricmagneticfield6 path
struct Species {
  double *pos[3], *vel[3];
  int64_t n[3];
  int64_t start[3];
};

struct EmState {
  double *x, *y, *z, *vx, *vy, *vz, *r, *phi, *vr, *q, *m, *E;
  int *del;
};

__device__ __forceinline__ int species_of(const Species &s, int64_t o) {
  return o >= s.start[2] ? 2 : (o >= s.start[1] ? 1 : 0);
}

// electricmagneticfield6.m:65-73, 113-118: concatenate the three species
__global__ void k_em_load(Species sp, EmState st, int64_t N, double e, double m_e, double m_i,
                          unsigned flags) {
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < N;
       o += (int64_t)gridDim.x * blockDim.x) {
    const int s = species_of(sp, o);
    const int64_t i = o - sp.start[s], ld = sp.n[s];
    const double p0 = sp.pos[s][i], p1 = sp.pos[s][ld + i], p2 = sp.pos[s][2 * ld + i];
    if (flags & GASATT_POS_IN_CYL) { st.x[o] = p0 * cos(p1); st.y[o] = p0 * sin(p1); }
    else { st.x[o] = p0; st.y[o] = p1; }
    st.z[o] = p2;
    st.vx[o] = sp.vel[s][i]; st.vy[o] = sp.vel[s][ld + i]; st.vz[o] = sp.vel[s][2 * ld + i];
    st.q[o] = s == 0 ? -e : (s == 1 ? e : 2 * e);
    st.m[o] = s == 0 ? m_e : m_i;
    st.r[o] = 0; st.phi[o] = 0; st.vr[o] = 0; st.E[o] = 0;
    st.del[o] = 0;
  }
}

// EM2.cu:23-57 then EM7.cu:51-202 for the same particle (the deposit of a
// particle needs only its own EM2 result)
__global__ void k_em2_deposit(EmState st, int64_t N, double Rp, double Lp, double PHIp,
                              double dt, int nr, int nz, double dr, double dz, double FN,
                              double scale, unsigned long long *Jr, unsigned long long *Jz,
                              unsigned flags) {
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < N;
       o += (int64_t)gridDim.x * blockDim.x) {
    if (st.del[o] == 1) continue;
    double x = st.x[o], y = st.y[o], z = st.z[o], vx = st.vx[o], vy = st.vy[o], vz = st.vz[o];
    double r, phi;
    int del = 0;
    halfdrift_cart(x, y, z, vx, vy, vz, vx, vy, vz, r, phi, del, Rp, Lp, PHIp, dt, flags);
    const double vr = vx * cos(phi) + vy * sin(phi);
    st.x[o] = x; st.y[o] = y; st.z[o] = z; st.vx[o] = vx; st.vy[o] = vy; st.vz[o] = vz;
    st.r[o] = r; st.phi[o] = phi; st.vr[o] = vr;
    if (del) { st.del[o] = 1; continue; }
    int64_t a[4]; double b[4];
    em7_weights(r, z, nr, nz, dr, dz, a, b);
    const double q = st.q[o];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      fx_add(Jr, a[k], FN * b[k] * q * vr, scale);
      fx_add(Jz, a[k], FN * b[k] * q * vz, scale);
    }
  }
}

// EM4.cu:33-177
__global__ void k_em4(EmState st, int64_t N, const double *Er, const double *Ez, const double *H,
                      double Rp, double Lp, double PHIp, int nr, int nz, double mu, double c,
                      double dr, double dz, double dt, unsigned flags) {
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < N;
       o += (int64_t)gridDim.x * blockDim.x) {
    if (st.del[o] == 1) continue;
    double Er0, Ez0, H0;
    gather3<double>(Er, Ez, H, nr, nz, dr, dz, st.r[o], st.z[o], Er0, Ez0, H0);
    const double vx = st.vx[o], vy = st.vy[o], vz = st.vz[o], q = st.q[o], m = st.m[o];
    const double phi = st.phi[o];
    double gamma = 1 / sqrt(1 - (vx * vx + vy * vy + vz * vz) / (c * c));
    double ux, uy, uz;
    if (flags & GASATT_Q_EULER_KICK) {
      const double Fr = q * (Er0 + (-vz * H0 * mu));
      const double Fz = q * (Ez0 + (st.vr[o] * H0 * mu));
      const double Fx = Fr * cos(phi), Fy = Fr * sin(phi);
      ux = gamma * vx + Fx / m * dt;
      uy = gamma * vy + Fy / m * dt;
      uz = gamma * vz + Fz / m * dt;
    } else {
      const double cp = cos(phi), sp = sin(phi);
      ux = gamma * vx; uy = gamma * vy; uz = gamma * vz;
      const double B = mu * H0;
      boris(ux, uy, uz, Er0 * cp, Er0 * sp, Ez0, -B * sp, B * cp, 0.0, q / m * dt / 2, c);
    }
    gamma = sqrt(1 + (ux * ux + uy * uy + uz * uz) / (c * c));
    st.E[o] = (gamma - 1) * m * c * c;
    double nvx = ux / gamma, nvy = uy / gamma, nvz = uz / gamma;
    double x = st.x[o], y = st.y[o], z = st.z[o], r, ph;
    int del = 0;
    halfdrift_cart(x, y, z, nvx, nvy, nvz, nvx, nvy, nvz, r, ph, del, Rp, Lp, PHIp, dt, flags);
    st.x[o] = x; st.y[o] = y; st.z[o] = z;
    st.vx[o] = nvx; st.vy[o] = nvy; st.vz[o] = nvz;
    st.r[o] = r; st.phi[o] = ph;
    if (del) st.del[o] = 1;
  }
}

__global__ void k_keep_flags(const int *del, int64_t N, int *keep) {
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o <= N;
       o += (int64_t)gridDim.x * blockDim.x)
    keep[o] = (o < N && del[o] == 0) ? 1 : 0;
}

// electricmagneticfield6.m:168-188 with each species compacted by its own
// delete flags; pos[] is the exclusive scan of the keep flags (N+1 entries)
__global__ void k_em_store(Species sp, EmState st, int64_t N, const int *pos, double *kin,
                           double e) {
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < N;
       o += (int64_t)gridDim.x * blockDim.x) {
    if (st.del[o]) continue;
    const int s = species_of(sp, o);
    const int64_t w = pos[o] - pos[sp.start[s]], ld = sp.n[s];
    sp.pos[s][w] = st.x[o]; sp.pos[s][ld + w] = st.y[o]; sp.pos[s][2 * ld + w] = st.z[o];
    sp.vel[s][w] = st.vx[o]; sp.vel[s][ld + w] = st.vy[o]; sp.vel[s][2 * ld + w] = st.vz[o];
    if (s == 0 && kin) kin[w] = st.E[o] / (1000 * e);
  }
}

// ------------------------------------------------------- electron_collision
struct MccTables {
  const double *xI, *yI, *V;  int ne;
  const double *exc;  int n_exc;     // n_exc x 5 column-major
  const double *dphi; const int *sum_cell0; int rmax; int cellnumxy;
  const double *density, *temperature; int64_t ncell;
};

__device__ __forceinline__ double pdf_k(const double *V, int ne, int i, int k, double a0,
                                        double b0, double TCS, double pi) {
  int64_t i1 = (int64_t)i * 181 + k, i2 = (int64_t)(i + 1) * 181 + k;
  const int64_t last = (int64_t)ne * 181 - 1;
  if (i1 > last) i1 = last;
  if (i2 > last) i2 = last;
  const double vI = a0 * V[i1] + b0 * V[i2];
  double D = exp(vI);
  D = 2 * pi * sin(k * pi / 180) * D * 2;
  return 1 / TCS * D;
}

// electron_transport.cu:88-121 (GASATT_Q_CDF_NEXTBIN) or get_ElasticSc_sub1.m
__device__ double elastic_theta(double energy, const MccTables &t, double U, double pi,
                                unsigned flags) {
  const double *xI = t.xI;
  const int ne = t.ne;
  double Ee = (flags & GASATT_Q_XS_LINEAR_E) ? energy : log(energy);
  if (!(flags & GASATT_Q_XS_LINEAR_E)) {
    if (Ee < xI[0]) Ee = xI[0];
    if (Ee > xI[ne - 1]) Ee = xI[ne - 1];
  }
  int i = 0;
  while (i < ne - 2 && Ee > xI[i + 1]) i++;
  const double a0 = (xI[i + 1] - Ee) / (xI[i + 1] - xI[i]);
  const double b0 = (Ee - xI[i]) / (xI[i + 1] - xI[i]);
  const double TCS = (a0 * t.yI[i] + b0 * t.yI[i + 1]) * 2;
  if (flags & GASATT_Q_CDF_NEXTBIN) {
    double imax = 0;
    for (int k = 0; k <= 180; ++k) imax = imax + pdf_k(t.V, ne, i, k, a0, b0, TCS, pi) * pi / 180;
    const double rnd = U * imax;
    double i1 = 0;
    int k = 0;
    while (rnd > i1 && k < 181) {
      i1 = i1 + pdf_k(t.V, ne, i, k, a0, b0, TCS, pi) * pi / 180;
      k++;
    }
    const double i2 = i1 + pdf_k(t.V, ne, i, k, a0, b0, TCS, pi) * pi / 180;
    const double aa = (i2 - rnd) / (i2 - i1), bb = (rnd - i1) / (i2 - i1);
    return (aa * (k - 1) + bb * k) * pi / 180;
  }
  // trapezoid CDF and linear inverse (cumtrapz + interp1)
  const double h = pi / 180;
  double C = 0, prev = pdf_k(t.V, ne, i, 0, a0, b0, TCS, pi);
  double tot = 0;
  {
    double p0 = prev;
    for (int k = 1; k <= 180; ++k) {
      const double pk = pdf_k(t.V, ne, i, k, a0, b0, TCS, pi);
      tot = tot + (p0 + pk) / 2 * h;
      p0 = pk;
    }
  }
  const double rn = U * tot;
  for (int k = 1; k <= 180; ++k) {
    const double pk = pdf_k(t.V, ne, i, k, a0, b0, TCS, pi);
    const double Cn = C + (prev + pk) / 2 * h;
    if (Cn > rn || k == 180) return ((k - 1) + (rn - C) / (Cn - C)) * h;
    C = Cn;
    prev = pk;
  }
  return pi;
}

__device__ __forceinline__ double pow_sel(double a, double b, unsigned flags) {
  if (flags & GASATT_Q_EXC_POWF) return (double)powf((float)a, (float)b);
  return pow(a, b);
}

struct MccOut {
  uint8_t *sec;
  double *svx, *svy, *svz, *sample, *ivx, *ivy, *ivz;
};

// electron_transport.cu:39-229; positions/velocities column-major (ld = cap)
__global__ void k_electron_transport(double *pos, double *vel, int64_t cap, int64_t n,
                                     const double *sig_el, const double *sig_ion,
                                     const double *sig_exc, const double *energy, MccTables t,
                                     MccOut out, double dr, double dz, double dt,
                                     const double *draws, uint64_t seed, int64_t call,
                                     unsigned flags) {
  const double e = GASATT_MCC_E, c = GASATT_MCC_C, m = GASATT_MCC_ME, m_ion = GASATT_MCC_MION;
  const double kb = GASATT_MCC_KB, E_e = m * c * c / e;
  const double pi = (flags & GASATT_Q_PI7) ? GASATT_MCC_PI7 : GASATT_PI;
  const double I = GASATT_ION_I_EV;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    out.sec[p] = 0;
    double U[GASATT_MCC_NDRAW];
    if (draws) {
#pragma unroll
      for (int k = 0; k < GASATT_MCC_NDRAW; ++k) U[k] = draws[p * GASATT_MCC_NDRAW + k];
    } else {
      U2 a = draw2(seed, (uint64_t)p, call, 0), b = draw2(seed, (uint64_t)p, call, 1);
      U2 g1 = draw2(seed, (uint64_t)p, call, 2), g2 = draw2(seed, (uint64_t)p, call, 3);
      U[0] = a.a; U[1] = a.b; U[2] = b.a; U[3] = b.b;
      const double rad1 = sqrt(-2 * log(g1.a)), rad2 = sqrt(-2 * log(g2.a));
      U[4] = rad1 * cos(2 * GASATT_PI * g1.b);
      U[5] = rad1 * sin(2 * GASATT_PI * g1.b);
      U[6] = rad2 * cos(2 * GASATT_PI * g2.b);
      U[7] = 0;
    }
    double vx = vel[p], vy = vel[cap + p], vz = vel[2 * cap + p];
    const double x = pos[p], y = pos[cap + p], z = pos[2 * cap + p];
    const double v_e = sqrt(vx * vx + vy * vy + vz * vz);
    const double dx = v_e * dt;
    const double r = sqrt(x * x + y * y);
    const double phi = atan(y / x);
    int iz = (int)floor(z / dz), ir = (int)floor(r / dr);
    if (ir > t.rmax - 1) ir = t.rmax - 1;
    if (ir < 0) ir = 0;
    int iphi = (int)floor(phi / t.dphi[ir]);
    const int nphi = t.sum_cell0[ir + 1] - t.sum_cell0[ir];
    if (iphi > nphi - 1) iphi = nphi - 1;
    if (iphi < 0) iphi = 0;
    int64_t index = (int64_t)iz * t.cellnumxy + t.sum_cell0[ir] + iphi;
    if (index < 0) index = 0;
    if (index > t.ncell - 1) index = t.ncell - 1;
    const double p_el = dx * t.density[index] * sig_el[p];
    const double p_io = dx * t.density[index] * sig_ion[p];
    const double p_ex = dx * t.density[index] * sig_exc[p];
    double p_tot = p_el + p_io + p_ex;
    const double a = p_el / p_tot;
    const double b = a + p_io / p_tot;
    if (!(flags & GASATT_Q_COLL_LINEAR_P)) p_tot = -expm1(-p_tot);
    if (!(U[0] < p_tot)) continue;
    const double en = energy[p];
    if (U[1] < a) {
      const double th = elastic_theta(en, t, U[2], pi, flags);
      const double ph = 2 * pi * U[3];
      rotate_v(vx, vy, vz, th, ph, true);
    } else if (U[1] < b && en > I / 1000) {
      const double T = en * 1000;
      const double T_a = 1000, T_b = 2 * I, t_b = I, T_s = 4.17, t_s = 13.8;
      const double T_0 = T_s - T_a / (T + T_b);
      const double tt = t_s * T / (T + t_b);
      const double T_m = (T - I) / 2;
      const double k_1 = atan((T_m - T_0) / tt);
      const double k_2 = atan(T_0 / tt);
      const double k0 = T_0 + tt * tan(U[2] * (k_1 + k_2) - k_2);
      const double E_1 = k0, E_2 = T - E_1 - I;
      double E_p, E_s;
      if (E_2 > E_1) { E_p = E_2; E_s = E_1; } else { E_p = E_1; E_s = E_2; }
      const double kk = (flags & GASATT_Q_SEC_LAB_FRAME) ? k0 : E_s;
      E_p = E_p * e;
      E_s = E_s * e;
      const double phi_p = 2 * pi * U[3];
      const double phi_s = phi_p - pi;
      const double th_p = asin(sqrt((kk / T) / ((1 - kk / T) * T / (2 * E_e) + 1)));
      const double th_s = asin(sqrt((1 - kk / T) / (1 + kk / (2 * E_e))));
      const double ix = vx / v_e, iy = vy / v_e, iz_ = vz / v_e;
      double gamma = 1 + E_p / (m * c * c);
      const double v_p = c * sqrt(1 - 1 / (gamma * gamma));
      const double ratio = v_p / v_e;
      vx = ratio * vx; vy = ratio * vy; vz = ratio * vz;
      rotate_v(vx, vy, vz, th_p, phi_p, true);
      gamma = 1 + E_s / (m * c * c);
      const double v_s = c * sqrt(1 - 1 / (gamma * gamma));
      out.sec[p] = 1;
      if (flags & GASATT_Q_SEC_LAB_FRAME) {
        out.svx[p] = v_s * sin(th_s) * cos(phi_s);
        out.svy[p] = v_s * sin(th_s) * sin(phi_s);
        out.svz[p] = v_s * cos(th_s);
      } else {
        double sx = ix * v_s, sy = iy * v_s, sz = iz_ * v_s;
        rotate_v(sx, sy, sz, th_s, phi_s, true);
        out.svx[p] = sx; out.svy[p] = sy; out.svz[p] = sz;
      }
      out.sample[p] = (double)index;
      const double sd = sqrt(m_ion / (kb * t.temperature[index]));
      out.ivx[p] = (double)(float)U[4] / sd;
      out.ivy[p] = (double)(float)U[5] / sd;
      out.ivz[p] = (double)(float)U[6] / sd;
    } else {
      const double T = en * 1000;
      double k1 = 0, k2 = 0;
      for (int i = 0; i < t.n_exc; ++i) {
        const double k = t.exc[i], A = t.exc[t.n_exc + i], om = t.exc[2 * t.n_exc + i];
        const double nu = t.exc[3 * t.n_exc + i], ga = t.exc[4 * t.n_exc + i];
        if (!(flags & GASATT_Q_EXC_POWF) && !(T > k)) continue;
        const double aE = GASATT_MCC_Q0 * A / (k * k);
        const double bE = pow_sel(k / T, om, flags);
        const double cE = pow_sel(pow_sel(1 - k / T, ga, flags), nu, flags);
        k1 = k1 + aE * bE * cE * k;
        k2 = k2 + aE * bE * cE;
      }
      if (k2 == 0) continue;
      const double E_dep = k1 / k2;
      const double E_p = T - E_dep;
      const double gamma = 1 + E_p * e / (m * c * c);
      const double v_p = c * sqrt(1 - 1 / (gamma * gamma));
      const double ratio = v_p / v_e;
      vx = ratio * vx; vy = ratio * vy; vz = ratio * vz;
    }
    vel[p] = vx; vel[cap + p] = vy; vel[2 * cap + p] = vz;
  }
}

__global__ void k_u8_to_int(const uint8_t *a, int64_t n, int *b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = i < n ? (int)a[i] : 0;
}

// electron_collision.m:63-75: append secondaries and ions in parent order
__global__ void k_append(double *e_pos, double *e_vel, int64_t cap_e, int64_t n_e,
                         double *i_pos, double *i_vel, int64_t cap_i, int64_t n_i,
                         const int *pos, MccOut out) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n_e;
       p += (int64_t)gridDim.x * blockDim.x) {
    if (!out.sec[p]) continue;
    const int64_t we = n_e + pos[p], wi = n_i + pos[p];
    for (int d = 0; d < 3; ++d) {
      const double v = e_pos[d * cap_e + p];
      e_pos[d * cap_e + we] = v;
      i_pos[d * cap_i + wi] = v;
    }
    e_vel[we] = out.svx[p]; e_vel[cap_e + we] = out.svy[p]; e_vel[2 * cap_e + we] = out.svz[p];
    i_vel[wi] = out.ivx[p]; i_vel[cap_i + wi] = out.ivy[p]; i_vel[2 * cap_i + wi] = out.ivz[p];
  }
}

int exclusive_scan(gasatt_ctx *ctx, const int *in, int *out, int64_t n, void *tmp, size_t tmp_bytes) {
  size_t need = 0;
  GASATT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, need, in, out, (int)n, ctx->stream));
  if (need > tmp_bytes) return fail(ctx, GASATT_E_ARG, "scan scratch too small");
  GASATT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(tmp, need, in, out, (int)n, ctx->stream));
  ctx->launches++;
  return GASATT_OK;
}

size_t scan_tmp_bytes(int64_t n) {
  size_t need = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, need, (const int *)nullptr, (int *)nullptr, (int)n);
  return need + 256;
}

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// device copy of a host array into a carved scratch region
struct Carver {
  char *base; size_t off = 0;
  template <typename T> T *take(size_t n) {
    T *p = (T *)(base + off);
    off += align256(n * sizeof(T));
    return p;
  }
};

}  // namespace

// ====================================================================== C ABI
extern "C" {

int gasatt_find_CS0(gasatt_ctx *ctx, const gasatt_tables *tab, const double *E_keV, int64_t n,
                    double *sig_el, double *sig_ion, double *sig_exc, unsigned flags) {
  if (!ctx) return GASATT_E_ARG;
  std::string err;
  int st = check_tables(tab, err);
  if (st) return fail(ctx, st, err);
  if (n < 0 || (n > 0 && (!E_keV || !sig_el || !sig_ion || !sig_exc)))
    return fail(ctx, GASATT_E_ARG, "find_CS0: bad arrays");
  if (n == 0) return GASATT_OK;
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t ne = 2 * (size_t)tab->n_el, ns = 2 * (size_t)tab->n_sel, ni = 2 * (size_t)tab->n_ion,
               nx = 5 * (size_t)tab->n_exc;
  void *buf;
  st = scratch(ctx, align256(ne * 8) + align256(ns * 8) + align256(ni * 8) + align256(nx * 8), &buf);
  if (st) return st;
  Carver cv{(char *)buf};
  double *d_el = cv.take<double>(ne), *d_sel = cv.take<double>(ns), *d_ion = cv.take<double>(ni),
         *d_exc = cv.take<double>(nx);
  GASATT_CUDA(ctx, cudaMemcpyAsync(d_el, tab->t_el, ne * 8, cudaMemcpyHostToDevice, ctx->stream));
  GASATT_CUDA(ctx, cudaMemcpyAsync(d_sel, tab->t_sel, ns * 8, cudaMemcpyHostToDevice, ctx->stream));
  GASATT_CUDA(ctx, cudaMemcpyAsync(d_ion, tab->t_ion, ni * 8, cudaMemcpyHostToDevice, ctx->stream));
  GASATT_CUDA(ctx, cudaMemcpyAsync(d_exc, tab->t_exc, nx * 8, cudaMemcpyHostToDevice, ctx->stream));
  XsRaw t{d_el, tab->n_el, d_sel, tab->n_sel, d_ion, tab->n_ion, d_exc, tab->n_exc};
  k_find_cs0<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(t, E_keV, n, sig_el, sig_ion, sig_exc, flags);
  GASATT_LAUNCHED(ctx);
  GASATT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GASATT_OK;
}

int gasatt_free_motion(gasatt_ctx *ctx, const double *vx, const double *vy, const double *vz,
                       const double *x, const double *y, const double *z, int64_t n, double dt,
                       double *xn, double *yn, double *zn, double *rn, double *phin) {
  if (!ctx || n < 0) return GASATT_E_ARG;
  if (n == 0) return GASATT_OK;
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  k_free_motion<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(vx, vy, vz, x, y, z, n, dt, xn, yn, zn, rn, phin);
  GASATT_LAUNCHED(ctx);
  return GASATT_OK;
}

int gasatt_rebond(gasatt_ctx *ctx, double *pos, int64_t ld_pos, const double *r,
                  const double *phi, double *vel, int64_t ld_vel, int64_t n, double Lp,
                  double PHIp, int64_t *n_boundary) {
  if (!ctx || n < 0 || ld_pos < n || ld_vel < n || !(PHIp > 0) || !(Lp > 0))
    return fail(ctx, GASATT_E_ARG, "REBOND: bad sizes");
  if (n_boundary) *n_boundary = 0;
  if (n == 0) return GASATT_OK;
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  void *buf;
  int st = scratch(ctx, 16, &buf);
  if (st) return st;
  unsigned long long *cnt = (unsigned long long *)buf, h[2] = {0, 0};
  GASATT_CUDA(ctx, cudaMemsetAsync(cnt, 0, 16, ctx->stream));
  // cos and sin of the wedge angle on the host, once, like the reference's
  // cos(PHIp) and sin(PHIp) of every wrap
  k_rebond<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(pos, ld_pos, r, phi, vel, ld_vel, n, Lp,
                                                             PHIp, std::cos(PHIp), std::sin(PHIp), cnt);
  GASATT_LAUNCHED(ctx);
  GASATT_CUDA(ctx, cudaMemcpyAsync(h, cnt, 16, cudaMemcpyDeviceToHost, ctx->stream));
  GASATT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (h[1]) return fail(ctx, GASATT_E_ARG, "REBOND: an azimuth lies more than 4096 wedges outside");
  if (n_boundary) *n_boundary = (int64_t)h[0];
  return GASATT_OK;
}

int gasatt_particle_density(gasatt_ctx *ctx, double dr, double dz, const double *dphi, int rmax,
                            const double *r, const double *phi, const double *z, int64_t n,
                            int cellnumxy, const double *sum_cell, const double *VC, int64_t ncell,
                            double FN, double *density) {
  if (!ctx || n < 0 || ncell <= 0 || rmax <= 0 || cellnumxy <= 0)
    return fail(ctx, GASATT_E_ARG, "particle_density: bad sizes");
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  void *buf;
  int st = scratch(ctx, (size_t)ncell * 8, &buf);
  if (st) return st;
  unsigned long long *cnt = (unsigned long long *)buf;
  GASATT_CUDA(ctx, cudaMemsetAsync(cnt, 0, (size_t)ncell * 8, ctx->stream));
  if (n > 0) {
    k_density_count<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(dr, dz, dphi, rmax, r, phi, z, n,
                                                                     cellnumxy, sum_cell, ncell, cnt);
    GASATT_LAUNCHED(ctx);
  }
  k_density_finish<<<grid_for(ncell, kBlock), kBlock, 0, ctx->stream>>>(cnt, ncell, cellnumxy, VC, FN, density);
  GASATT_LAUNCHED(ctx);
  return GASATT_OK;
}

int gasatt_particle_density_noalloc(gasatt_ctx *ctx, double dr, double dz, const double *dphi,
                                    int rmax, const double *r, const double *phi, const double *z,
                                    int64_t n, int cellnumxy, const double *sum_cell,
                                    const double *VC, int64_t ncell, double FN, double *density) {
  if (!ctx || n < 0 || ncell <= 0 || rmax <= 0 || cellnumxy <= 0)
    return fail(ctx, GASATT_E_ARG, "particle_density_noalloc: bad sizes");
  if (ncell > (int64_t)GASATT_DENSITY_NOALLOC_MAX_CELLS)
    return fail(ctx, GASATT_E_CAPACITY,
                "particle_density_noalloc: ncell = " + std::to_string(ncell) +
                    " exceeds its fixed scratch of " +
                    std::to_string((long long)GASATT_DENSITY_NOALLOC_MAX_CELLS) +
                    " cells (use gasatt_particle_density)");
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  unsigned long long *cnt = nullptr;
  int st = density_counts_on_device(ctx, &cnt);
  if (st) return st;
  // the array keeps the previous call's counts: clear the cells used now
  GASATT_CUDA(ctx, cudaMemsetAsync(cnt, 0, (size_t)ncell * 8, ctx->stream));
  if (n > 0) {
    k_density_count<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(dr, dz, dphi, rmax, r, phi, z, n,
                                                                     cellnumxy, sum_cell, ncell, cnt);
    GASATT_LAUNCHED(ctx);
  }
  k_density_finish<<<grid_for(ncell, kBlock), kBlock, 0, ctx->stream>>>(cnt, ncell, cellnumxy, VC, FN, density);
  GASATT_LAUNCHED(ctx);
  return GASATT_OK;
}

int gasatt_electricmagneticfield6(gasatt_ctx *ctx, double *e_pos, double *e_vel, int64_t n_e,
                                  double *i1_pos, double *i1_vel, int64_t n_i1, double *i2_pos,
                                  double *i2_vel, int64_t n_i2, double *Er, double *Ez,
                                  double *Hphi, int n_r, int n_z, double delta, double dt,
                                  double Rp, double Lp, double PHIp, double FN, int cycle_time,
                                  double *electron_kinetic, int64_t *n_e_out, int64_t *n_i1_out,
                                  int64_t *n_i2_out, unsigned flags) {
  if (!ctx) return GASATT_E_ARG;
  if (n_e < 0 || n_i1 < 0 || n_i2 < 0 || n_r < 1 || n_z < 2 || !(delta > 0) || cycle_time < 0)
    return fail(ctx, GASATT_E_ARG, "electricmagneticfield6: bad sizes");
  if (std::fabs(Rp / delta - n_r) > 1e-6 * n_r || std::fabs(Lp / delta - n_z) > 1e-6 * n_z)
    return fail(ctx, GASATT_E_ARG, "electricmagneticfield6: grid must be Rp/delta x Lp/delta");
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  const int64_t N = n_e + n_i1 + n_i2;
  const int64_t ncel = (int64_t)n_r * n_z;
  const size_t sc = scan_tmp_bytes(N + 1);
  const size_t bytes = 12 * align256((size_t)(N + 1) * 8) + 3 * align256((size_t)(N + 1) * 4) +
                       2 * align256((size_t)ncel * 8) + align256(sc);
  void *buf;
  int st = scratch(ctx, bytes, &buf);
  if (st) return st;
  Carver cv{(char *)buf};
  EmState s;
  double **f[12] = {&s.x, &s.y, &s.z, &s.vx, &s.vy, &s.vz, &s.r, &s.phi, &s.vr, &s.q, &s.m, &s.E};
  for (int i = 0; i < 12; ++i) *f[i] = cv.take<double>(N + 1);
  s.del = cv.take<int>(N + 1);
  int *keep = cv.take<int>(N + 1), *scanned = cv.take<int>(N + 1);
  unsigned long long *Jr = cv.take<unsigned long long>(ncel), *Jz = cv.take<unsigned long long>(ncel);
  void *tmp = cv.take<char>(sc);
  Species sp;
  sp.pos[0] = e_pos; sp.pos[1] = i1_pos; sp.pos[2] = i2_pos;
  sp.vel[0] = e_vel; sp.vel[1] = i1_vel; sp.vel[2] = i2_vel;
  sp.n[0] = n_e; sp.n[1] = n_i1; sp.n[2] = n_i2;
  sp.start[0] = 0; sp.start[1] = n_e; sp.start[2] = n_e + n_i1;
  const double e = GASATT_EM_E, c = GASATT_EM_C, mu = GASATT_EM_MU, eps = GASATT_EM_EPS;
  const unsigned g = grid_for(N, kBlock);
  if (N > 0) {
    k_em_load<<<g, kBlock, 0, ctx->stream>>>(sp, s, N, e, GASATT_EM_ME, GASATT_EM_MION, flags);
    GASATT_LAUNCHED(ctx);
  }
  // fixed-point scale: |q FN v w| <= 2e FN c per particle, N particles per node at most
  const double bound = (double)(N > 0 ? N : 1) * 2 * e * std::fabs(FN) * c;
  const int S = (int)std::floor(std::log2(std::ldexp(1.0, 62) / bound));
  const double scale = std::ldexp(1.0, S);
  const int ratio = 5;
  const double ddt = ratio * dt;                       // electricmagneticfield6.m:134-135
  FdtdCoef fc;
  fc.dr = delta; fc.dz = delta; fc.PHIp = PHIp; fc.inv_scale = std::ldexp(1.0, -S);
  fc.dt_eps = (dt / 2) / eps;
  fc.dt_eps_dz = (dt / 2) / (eps * delta);
  fc.axis = 4 * (dt / 2) / (eps * delta);
  const unsigned gh = grid_for(ncel, kBlock), ge = grid_for((int64_t)(n_r + 1) * (n_z + 1), kBlock);
  for (int k = 0; k < cycle_time / ratio; ++k) {        // :138-166
    GASATT_CUDA(ctx, cudaMemsetAsync(Jr, 0, (size_t)ncel * 8, ctx->stream));
    GASATT_CUDA(ctx, cudaMemsetAsync(Jz, 0, (size_t)ncel * 8, ctx->stream));
    if (N > 0) {
      k_em2_deposit<<<g, kBlock, 0, ctx->stream>>>(s, N, Rp, Lp, PHIp, ddt, n_r, n_z, delta, delta,
                                                   FN, scale, Jr, Jz, flags);
      GASATT_LAUNCHED(ctx);
    }
    const double hdt[3] = {-dt / 4, dt / 2, dt / 4};
    auto hstep = [&](double h) {
      k_fdtd_h<double><<<gh, kBlock, 0, ctx->stream>>>(Hphi, Er, Ez, n_r, n_z, h / (mu * delta),
                                                      h / (mu * delta));
    };
    hstep(hdt[0]);
    GASATT_LAUNCHED(ctx);
    for (int i = 0; i < 2 * ratio; ++i) {
      hstep(hdt[1]);
      GASATT_LAUNCHED(ctx);
      k_fdtd_e<double><<<ge, kBlock, 0, ctx->stream>>>(Er, Ez, Hphi, Jr, Jz, n_r, n_z, fc, flags);
      GASATT_LAUNCHED(ctx);
    }
    hstep(hdt[2]);
    GASATT_LAUNCHED(ctx);
    if (N > 0) {
      k_em4<<<g, kBlock, 0, ctx->stream>>>(s, N, Er, Ez, Hphi, Rp, Lp, PHIp, n_r, n_z, mu, c, delta,
                                           delta, ddt, flags);
      GASATT_LAUNCHED(ctx);
    }
  }
  int64_t outs[3] = {0, 0, 0};
  if (N > 0) {
    k_keep_flags<<<grid_for(N + 1, kBlock), kBlock, 0, ctx->stream>>>(s.del, N, keep);
    GASATT_LAUNCHED(ctx);
    st = exclusive_scan(ctx, keep, scanned, N + 1, tmp, sc);
    if (st) return st;
    k_em_store<<<g, kBlock, 0, ctx->stream>>>(sp, s, N, scanned, electron_kinetic, e);
    GASATT_LAUNCHED(ctx);
    int h[4];
    const int64_t idx[4] = {0, n_e, n_e + n_i1, N};
    for (int i = 0; i < 4; ++i)
      GASATT_CUDA(ctx, cudaMemcpyAsync((int *)ctx->pinned + i, scanned + idx[i], 4,
                                       cudaMemcpyDeviceToHost, ctx->stream));
    GASATT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::memcpy(h, ctx->pinned, sizeof(h));
    outs[0] = h[1] - h[0]; outs[1] = h[2] - h[1]; outs[2] = h[3] - h[2];
  } else {
    GASATT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  if (n_e_out) *n_e_out = outs[0];
  if (n_i1_out) *n_i1_out = outs[1];
  if (n_i2_out) *n_i2_out = outs[2];
  return GASATT_OK;
}

int gasatt_electron_collision(gasatt_ctx *ctx, double *e_pos, double *e_vel, int64_t n_e,
                              int64_t cap_e, double *i1_pos, double *i1_vel, int64_t n_i1,
                              int64_t cap_i1, const gasatt_tables *tab,
                              const double *electron_kinetic, const double *sum_cell, int rmax,
                              int cellnumxy, const double *density, const double *temperature,
                              int64_t ncell, double PHIp, const double *phimax, double dr,
                              double dz, const double *sig_el, const double *sig_ion,
                              const double *sig_exc, double dt_transport, const double *draws,
                              int64_t *n_e_out, int64_t *n_i1_out, unsigned flags) {
  if (!ctx) return GASATT_E_ARG;
  if (n_e < 0 || cap_e < n_e || n_i1 < 0 || cap_i1 < n_i1 || rmax < 1 || cellnumxy < 1 || ncell < 1)
    return fail(ctx, GASATT_E_ARG, "electron_collision: bad sizes");
  ElasticTables el;
  std::string err;
  int st = build_elastic_tables(tab, el, err);
  if (st) return fail(ctx, st, err);
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  std::vector<int> sc0(rmax + 1);
  std::vector<double> dphi(rmax);
  sc0[0] = 0;                                           // electron_collision.m:53-54
  for (int i = 0; i < rmax; ++i) { sc0[i + 1] = (int)sum_cell[i]; dphi[i] = PHIp * 1 / phimax[i]; }
  const int64_t n = n_e;
  const size_t sc = scan_tmp_bytes(n + 1);
  const size_t bytes = align256(el.xInterp.size() * 8) * 2 + align256(el.V.size() * 8) +
                       align256((size_t)5 * tab->n_exc * 8) + align256((size_t)rmax * 8) +
                       align256((size_t)(rmax + 1) * 4) + align256((size_t)(n + 1)) +
                       7 * align256((size_t)(n + 1) * 8) + 2 * align256((size_t)(n + 1) * 4) +
                       align256(sc);
  void *buf;
  st = scratch(ctx, bytes, &buf);
  if (st) return st;
  Carver cv{(char *)buf};
  double *d_xI = cv.take<double>(el.ne), *d_yI = cv.take<double>(el.ne), *d_V = cv.take<double>(el.V.size());
  double *d_exc = cv.take<double>(5 * tab->n_exc), *d_dphi = cv.take<double>(rmax);
  int *d_sc0 = cv.take<int>(rmax + 1);
  MccOut out;
  out.sec = cv.take<uint8_t>(n + 1);
  double **o7[7] = {&out.svx, &out.svy, &out.svz, &out.sample, &out.ivx, &out.ivy, &out.ivz};
  for (int i = 0; i < 7; ++i) *o7[i] = cv.take<double>(n + 1);
  int *flag_i = cv.take<int>(n + 1), *posb = cv.take<int>(n + 1);
  void *tmp = cv.take<char>(sc);
  cudaStream_t s = ctx->stream;
  GASATT_CUDA(ctx, cudaMemcpyAsync(d_xI, el.xInterp.data(), el.ne * 8, cudaMemcpyHostToDevice, s));
  GASATT_CUDA(ctx, cudaMemcpyAsync(d_yI, el.yInterp.data(), el.ne * 8, cudaMemcpyHostToDevice, s));
  GASATT_CUDA(ctx, cudaMemcpyAsync(d_V, el.V.data(), el.V.size() * 8, cudaMemcpyHostToDevice, s));
  GASATT_CUDA(ctx, cudaMemcpyAsync(d_exc, tab->t_exc, (size_t)5 * tab->n_exc * 8, cudaMemcpyHostToDevice, s));
  GASATT_CUDA(ctx, cudaMemcpyAsync(d_dphi, dphi.data(), (size_t)rmax * 8, cudaMemcpyHostToDevice, s));
  GASATT_CUDA(ctx, cudaMemcpyAsync(d_sc0, sc0.data(), (size_t)(rmax + 1) * 4, cudaMemcpyHostToDevice, s));
  MccTables t{d_xI, d_yI, d_V, el.ne, d_exc, tab->n_exc, d_dphi, d_sc0, rmax, cellnumxy,
              density, temperature, ncell};
  const int64_t call = ctx->mcc_calls++;
  if (n > 0) {
    k_electron_transport<<<grid_for(n, kBlock), kBlock, 0, s>>>(
        e_pos, e_vel, cap_e, n, sig_el, sig_ion, sig_exc, electron_kinetic, t, out, dr, dz,
        dt_transport, draws, ctx->seed, call, flags);
    GASATT_LAUNCHED(ctx);
  }
  k_u8_to_int<<<grid_for(n + 1, kBlock), kBlock, 0, s>>>(out.sec, n, flag_i);
  GASATT_LAUNCHED(ctx);
  st = exclusive_scan(ctx, flag_i, posb, n + 1, tmp, sc);
  if (st) return st;
  GASATT_CUDA(ctx, cudaMemcpyAsync(ctx->pinned, posb + n, 4, cudaMemcpyDeviceToHost, s));
  GASATT_CUDA(ctx, cudaStreamSynchronize(s));
  int nb;
  std::memcpy(&nb, ctx->pinned, 4);
  if (n_e + nb > cap_e || n_i1 + nb > cap_i1)
    return fail(ctx, GASATT_E_CAPACITY, "electron_collision: no room for the secondaries");
  if (n > 0 && nb > 0) {
    k_append<<<grid_for(n, kBlock), kBlock, 0, s>>>(e_pos, e_vel, cap_e, n_e, i1_pos, i1_vel,
                                                    cap_i1, n_i1, posb, out);
    GASATT_LAUNCHED(ctx);
  }
  GASATT_CUDA(ctx, cudaStreamSynchronize(s));
  if (n_e_out) *n_e_out = n_e + nb;
  if (n_i1_out) *n_i1_out = n_i1 + nb;
  return GASATT_OK;
}

}  // extern "C"
