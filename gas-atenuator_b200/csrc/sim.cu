// sim.cu - the resident PIC-MCC simulation (the hot path).
//
// One step s = FDTD sub-cycle (fields t^s -> t^{s+1}) followed by one fused
// particle pass:
//   gather (EM4.cu:41-122) -> relativistic Boris kick -> drift over the step
//   with the wall / end rules (EM2.cu:26-57, EM4.cu:146-177) -> current
//   deposit (EM7.cu:56-202) into 64-bit fixed point -> null-collision
//   candidate test,
// and then the null-collision MCC of the candidates against the tabulated N2
// cross-sections (electron_transport.cu:64-227, corrected) with secondary
// birth, at the end of the step (operator splitting: push, then collide, as
// the reference's driver alternates its push and electron_collision calls).
// That collision kernel touches neither fields nor current, so the step graph
// runs it beside the next field update; observations of the state (read,
// diagnostics, sort, end of a run) first apply any collisions still queued.
// Particles never leave HBM; the per-step sequence is replayed from CUDA graphs.
//
// Two state forms:
//   FP64      r, z [m]; u_r, u_theta, u_z = gamma v [m/s]; id.  Dead: r < 0.
//   FP32      key = (iz << 16) | ir, fr, fz in-cell offsets [cells], u / c
//             (gamma beta) in float; id.  Dead: key = 0xFFFFFFFF.
// The collision test, branch selection, energy sharing and threshold
// subtraction run in FP64 in both forms.
//
// Deposit: each particle's four node contributions (q FN v w) are rounded to
// integers first, so the grid sum is exact and independent of order.  FP32:
// a shared-memory window per chunk of sorted particles; FP64: lanes of a warp
// that hit the same four nodes (equal sort key) are summed with
// __reduce_add_sync before one 64-bit atomic per node.
//
// The FP32 form drifts the whole step at once (the reference's two half
// drifts joined).
#include <cmath>
#include <cstring>
#include <vector>
#include <cudaTypedefs.h>
#include "fdtd.cuh"
#include "fdtd_tma.cuh"
#include "gasatt_internal.h"

using namespace gasatt;

namespace {

constexpr uint32_t kDead = 0xFFFFFFFFu;
constexpr int kBlock = 256;
constexpr int kMccBlock = 64;             // collision kernels: two warps per block

// Device counters.  Fields that every thread reads when a kernel starts share
// the first 128-byte line; the counters that take atomics during a pass get
// lines of their own, so those atomics do not hold up the reads.
struct SimCounters {
  unsigned long long n_total;    // committed slots
  long long step;                // FP64: index of the next particle pass; FP32: of the current one
  unsigned long long cap;        // slot capacity
  unsigned long long sorted_total;
  long long cand_step[2];        // FP64: the pass that queued each queue
  int uncommitted;               // FP64: a pass ran since the last commit (k_commit)
  int pad0_;
  unsigned long long pad1_[9];
  unsigned long long n_births;   // slots claimed by births since the last commit
  unsigned long long pad2_[15];
  unsigned long long n_cand[2];  // collision candidates queued, per queue parity
  unsigned long long pad3_[14];
  unsigned long long chunk_next; // FP32 pass: next chunk to hand out
  unsigned long long pad4_[15];
  unsigned long long ion, ela, exc, nul, lost, cap_overflow;
  unsigned long long kin_fx;     // diagnostic: sum E_kin * 2^16 [eV]
  unsigned long long alive;      // diagnostic
  unsigned long long exc_loss_fx; // diagnostic: excitation energy losses * 2^16 [eV]
  unsigned long long wall_loss_fx;// diagnostic: kinetic energy absorbed at r = Rp * 2^16 [eV]
  unsigned fdtd_err;             // a field-update block gave up waiting for its tile copy
  unsigned scan_err;             // a sort's scan gave up waiting for a predecessor tile
  unsigned long long pad5_[5];
  unsigned long long n_ions;     // ion slots claimed (loads and births; may pass the capacity)
  unsigned long long ion_overflow, ion_lost;
  unsigned long long ion_alive, ion_charge, ion_kin_fx;   // diagnostics; kinetic: E * 2^32 [eV]
};

// slots holding particles, including births of the last pass not yet committed
__device__ __forceinline__ long long slots_in_use(const SimCounters *cnt) {
  const unsigned long long nt = cnt->n_total + cnt->n_births;
  return (long long)(nt < cnt->cap ? nt : cnt->cap);
}

// N2+ ions (FP64 in both forms): (r, z), (u_r, u_theta), u_z, id, charge number
struct IonState { double2 *rz; double2 *urt; double *uz; uint64_t *id; int8_t *q; };

struct SimParams {
  int nr, nz;
  int ldf, ldj;             // row strides (elements) of the field grids and of the current grids
  double dr, dz, dt, c, qe, me, mu0, FN, PHIp, n_gas, nu_max, P_null, Rp, Lp, kb, m_ion, T_gas;
  const double *gas;        // per-cell N2 density [m^-3] (n_r x n_z), or null: n_gas everywhere
  const double *ion_sig;    // per-cell sqrt(kT/m_ion) of newborn ions (n_r x n_z), or null: ion_sigma
  uint64_t seed;
  PhiloxKeys pk;            // Philox round keys of seed
  int secondaries;
  long long cap;
  double qm_dt2;            // -q_e/m_e dt/2
  float aE, aB, hdr, hdz;   // FP32 form: impulse per (V/m), per (A/m); c dt/(2 dr), c dt/(2 dz)
  double dep;               // fixed-point factor: FP64 q FN scale (x v)
  float depf;               // FP32: q FN c scale (x beta)
  uint64_t cand_below;      // null-collision candidate iff the 52-bit draw is below this
  int chunk;                // FP32 pass: particles per chunk (a multiple of the block, <= kChunkMax)
  // tables
  const double *sig;        // 3 x G (el, ion, exc)
  const double *cdf;        // G x 181
  const double *edep;       // G: mean excitation energy loss [eV]
  double exc_kmin;          // lowest excitation threshold [eV]
  int G;
  double lnEmin, dlnE;
  int n_exc;
  double exc[5][16];
  unsigned long long *Jr, *Jz;
  const float4 *qEr, *qEz, *qH;   // FP32 form: packed gather quads (FieldQuads)
  IonState ion;             // ion store (ion_cap > 0)
  long long ion_cap;        // ions stored at most; 0: no ion species
  double ion_sigma;         // spread of a newborn ion's velocity components sqrt(kT/m) [m/s]
};

template <typename Real>
struct Fields { Real *Er, *Ez, *H; };

// FP64: (r, z), (u_r, u_theta), u_z, id.   FP32: (key, fr, fz, u_r), (u_theta, u_z), id.
struct State64 { double2 *rz; double2 *urt; double *uz; uint64_t *id; };
struct State32 { uint4 *a; float2 *b; uint64_t *id; };

// ------------------------------------------------------------------- MCC
struct Birth { bool born; double ux, uy, uz; double eloss; };   // eloss: excitation loss [eV]

__device__ __forceinline__ void xs_lookup(const SimParams &P, double Eev, double &se, double &si,
                                          double &sx, double &L) {
  L = (log(Eev) - P.lnEmin) / P.dlnE;
  int i;
  double f;
  if (!(L > 0)) { i = 0; f = 0; }
  else if (L >= P.G - 1) { i = P.G - 2; f = 1; }
  else { i = (int)L; f = L - i; }
  const double *s0 = P.sig, *s1 = P.sig + P.G, *s2 = P.sig + 2 * P.G;
  se = s0[i] + f * (s0[i + 1] - s0[i]);
  si = s1[i] + f * (s1[i + 1] - s1[i]);
  sx = s2[i] + f * (s2[i + 1] - s2[i]);
}

// Inverse CDF: the largest k in [0, 179] with C[k] <= U, then linear in
// between (interp1 of the cumtrapz, get_ElasticSc_sub1.m:16-19).  Found in two
// rounds of independent loads (every 12th entry, then the 12 in the bracket)
// instead of eight dependent ones; same k as a bisection.
__device__ __forceinline__ double cdf_theta(const SimParams &P, double L, double U) {
  const double Lr = floor(L + 0.5);
  const int g = Lr < 0 ? 0 : (Lr > P.G - 1 ? P.G - 1 : (int)Lr);
  const double *C = P.cdf + (int64_t)g * 181;
  double coarse[15];
#pragma unroll
  for (int m = 0; m < 15; ++m) coarse[m] = C[12 * (m + 1)];
  int seg = 0;                                     // C[12 seg] <= U
#pragma unroll
  for (int m = 0; m < 15; ++m) seg += coarse[m] <= U ? 1 : 0;
  const int base = 12 * seg;
  double fine[12];
#pragma unroll
  for (int m = 0; m < 12; ++m) fine[m] = C[min(base + 1 + m, 180)];
  int lo = base;
#pragma unroll
  for (int m = 0; m < 12; ++m) lo += (base + 1 + m <= 179 && fine[m] <= U) ? 1 : 0;
  const double c0 = lo == base ? C[base] : fine[lo - base - 1];
  const double c1 = fine[lo - base];
  return (lo + (U - c0) / (c1 - c0)) * (GASATT_PI / 180);
}

__device__ __forceinline__ double u_of_energy(double EJ, double m, double c) {
  const double e = EJ / (m * c * c);
  return c * sqrt(e * (2 + e));
}

// Null-collision candidate test U1 < P_null on the integer draw: with
// U1 = (2b+1) 2^-53 (b the top 52 bits of the first two words) this is
// exactly b < P.cand_below.
__device__ __forceinline__ bool null_candidate(const SimParams &P, uint64_t id, long long step) {
  uint32_t c[4] = {(uint32_t)id, (uint32_t)(id >> 32), (uint32_t)step, 0u};
  philox4x32_10(c, P.pk);
  const uint64_t b = ((((uint64_t)c[0]) << 32) | c[1]) >> 12;
  return b < P.cand_below;
}

// Turn (vx, vy, vz) by the polar angle th and the azimuth ph about its own
// direction, from their sines and cosines (the rotation of
// electron_transport.cu:118-135 in the corrected frame, p2 = vx^2 + vy^2).
template <typename R>
__device__ __forceinline__ void rotate_sc(R &vx, R &vy, R &vz, R st, R ct, R sp, R cp) {
  const R v = sqrt(vx * vx + vy * vy + vz * vz);
  const R p2 = vx * vx + vy * vy;
  R x0, y0, z0;
  if (p2 > R(0.0001)) {
    const R s = sqrt(p2);
    const R f = st / s;
    x0 = vx * ct + f * (vx * vz * cp - v * vy * sp);
    y0 = vy * ct + f * (vy * vz * cp + v * vx * sp);
    z0 = vz * ct - s * st * cp;
  } else {
    x0 = v * st * cp;
    y0 = v * st * sp;
    z0 = v * ct;
  }
  vx = x0; vy = y0; vz = z0;
}

// Apply the rotation with (st, ct) given and azimuth 2 pi b (sign = -1: the
// opposite azimuth, phi - pi).  FAST (the FP32 form): float arithmetic with
// the hardware sine and cosine on the azimuth folded into [-pi, pi].
template <bool FAST>
__device__ __forceinline__ void turn(double &ux, double &uy, double &uz, double st, double ct,
                                     double b, double sign) {
  if (FAST) {
    float sp, cp;
    const float ph = (float)(2 * GASATT_PI * (b > 0.5 ? b - 1 : b));
    __sincosf(ph, &sp, &cp);
    float x = (float)ux, y = (float)uy, z = (float)uz;
    rotate_sc<float>(x, y, z, (float)st, (float)ct, (float)sign * sp, (float)sign * cp);
    ux = x; uy = y; uz = z;
  } else {
    double sp, cp;
    sincos(2 * GASATT_PI * b, &sp, &cp);
    rotate_sc<double>(ux, uy, uz, st, ct, sign * sp, sign * cp);
  }
}

// Collision of a candidate electron at step `step` (corrected form of
// electron_transport.cu:74-227).  u in m/s, local (r, theta, z) frame.
// Returns 1 elastic, 2 ionization, 3 excitation, 4 null.  The collision test,
// the branch choice, the ionization energy sharing and the threshold
// subtractions are FP64 in both forms; FAST (the FP32 form) turns the
// velocity in float.  The code is kept short: one candidate runs it alone,
// mostly from a cold instruction cache.
// gas density of cell (ir, iz), the neutral background of the collisions
__device__ __forceinline__ double gas_density(const SimParams &P, int ir, int iz) {
  if (!P.gas) return P.n_gas;
  ir = min(max(ir, 0), P.nr - 1);
  iz = min(max(iz, 0), P.nz - 1);
  return P.gas[ir + (int64_t)iz * P.nr];
}

// velocity spread sqrt(kT/m_ion) of an ion born in cell (ir, iz): the gas
// temperature of that cell (electron_transport.cu:202-204 reads
// temperature[index]) or the uniform one
__device__ __forceinline__ double ion_spread(const SimParams &P, int ir, int iz) {
  if (!P.ion_sig) return P.ion_sigma;
  ir = min(max(ir, 0), P.nr - 1);
  iz = min(max(iz, 0), P.nz - 1);
  return P.ion_sig[ir + (int64_t)iz * P.nr];
}

template <bool FAST>
__device__ __forceinline__ int mcc_event(const SimParams &P, uint64_t id, long long step, double &ux,
                                      double &uy, double &uz, Birth &b, double n_gas) {
  b.born = false;
  b.eloss = 0;
  const U2 d0 = draw2(P.seed, id, step, 0);
  const double c = P.c, me = P.me, qe = P.qe, I = GASATT_ION_I_EV;
  const double u2 = ux * ux + uy * uy + uz * uz;
  const double g = sqrt(1 + u2 / (c * c));
  const double EJ = me * c * c * ((u2 / (c * c)) / (g + 1));
  const double Eev = EJ / qe;
  const double um = sqrt(u2), v = um / g;
  double se, si, sx, L;
  xs_lookup(P, Eev, se, si, sx, L);
  const double nu_el = n_gas * se * v, nu_io = n_gas * si * v, nu_ex = n_gas * sx * v;
  const double X = d0.b * P.nu_max;
  if (X < nu_el) {
    const U2 d1 = draw2(P.seed, id, step, 1);
    const double th = cdf_theta(P, L, d1.a);
    double st, ct;
    if (FAST) {
      float sf, cf;
      __sincosf((float)th, &sf, &cf);
      st = sf; ct = cf;
    } else {
      sincos(th, &st, &ct);
    }
    turn<FAST>(ux, uy, uz, st, ct, d1.b, 1.0);
    return 1;
  }
  if (X < nu_el + nu_io && Eev > I) {
    const U2 d1 = draw2(P.seed, id, step, 1);
    const double T = Eev;
    const double T_a = 1000, T_b = 2 * I, t_b = I, T_s = 4.17, t_s = 13.8;
    const double T_0 = T_s - T_a / (T + T_b);
    const double t = t_s * T / (T + t_b);
    const double T_m = (T - I) / 2;
    // E_1 = T_0 + t tan(U (k_1 + k_2) - k_2), k_1 = atan((T_m - T_0)/t),
    // k_2 = atan(T_0/t): with k_1 + k_2 from one atan2 and
    // tan(x - k_2) = (tan x - tan k_2) / (1 + tan x tan k_2)
    const double a1 = (T_m - T_0) / t, a2 = T_0 / t;
    const double tx = tan(d1.a * atan2(a1 + a2, 1 - a1 * a2));
    const double k0 = T_0 + t * ((tx - a2) / (1 + a2 * tx));
    const double E_1 = k0, E_2 = T - E_1 - I;
    double E_p, E_s;
    if (E_2 > E_1) { E_p = E_2; E_s = E_1; } else { E_p = E_1; E_s = E_2; }
    const double E_e = me * c * c / qe;
    // polar angles as sines (the reference's asin arguments) and cosines
    const double sp2 = (E_s / T) / ((1 - E_s / T) * T / (2 * E_e) + 1);
    const double ss2 = (1 - E_s / T) / (1 + E_s / (2 * E_e));
    const double ix = ux / um, iy = uy / um, iz = uz / um;
    const double up = u_of_energy(E_p * qe, me, c), us = u_of_energy(E_s * qe, me, c);
    ux = ix * up; uy = iy * up; uz = iz * up;
    turn<FAST>(ux, uy, uz, sqrt(sp2), sqrt(1 - sp2), d1.b, 1.0);
    if (P.secondaries) {
      double sx_ = ix * us, sy_ = iy * us, sz_ = iz * us;
      turn<FAST>(sx_, sy_, sz_, sqrt(ss2), sqrt(1 - ss2), d1.b, -1.0);
      b.born = true; b.ux = sx_; b.uy = sy_; b.uz = sz_;
    }
    return 2;
  }
  if (X < nu_el + nu_io + nu_ex) {
    // tabulated mean energy loss, interpolated like the cross-sections
    if (!(Eev > P.exc_kmin)) return 4;
    int i;
    double f;
    if (!(L > 0)) { i = 0; f = 0; }
    else if (L >= P.G - 1) { i = P.G - 2; f = 1; }
    else { i = (int)L; f = L - i; }
    const double E_dep = P.edep[i] + f * (P.edep[i + 1] - P.edep[i]);
    if (!(E_dep > 0) || !(E_dep < Eev)) return 4;
    const double up = u_of_energy((Eev - E_dep) * qe, me, c);
    ux = ux / um * up; uy = uy / um * up; uz = uz / um * up;
    b.eloss = E_dep;
    return 3;
  }
  return 4;
}

// kinetic energy of a particle absorbed at the wall, u2 = |u / c|^2 and
// mc2 = m c^2 / q_e [eV] (rare: taken only on the step it leaves)
__device__ __forceinline__ void count_wall_loss(SimCounters *cnt, double u2, double mc2) {
  const double E = mc2 * (u2 / (sqrt(1 + u2) + 1));
  atomicAdd(&cnt->wall_loss_fx, (unsigned long long)__double2ll_rn(E * 65536.0));
}

__device__ __forceinline__ void count_event(SimCounters *cnt, int ev, const Birth &b) {
  if (ev == 1) atomicAdd(&cnt->ela, 1ull);
  else if (ev == 2) atomicAdd(&cnt->ion, 1ull);
  else if (ev == 3) {
    atomicAdd(&cnt->exc, 1ull);
    atomicAdd(&cnt->exc_loss_fx, (unsigned long long)__double2ll_rn(b.eloss * 65536.0));
  } else if (ev == 4) atomicAdd(&cnt->nul, 1ull);
}

// The N2+ ion of an ionization of electron `id` at step `step`, at the
// parent's position (r, z), singly charged, with a Maxwellian velocity at the
// gas temperature: each component normal with spread sqrt(kT/m)
// (electron_transport.cu:202-204).  The three normals are the Box-Muller
// transforms of the Philox draws (id, step) blocks 2 and 3; the ion takes the
// id of the secondary electron.  Takes no SimParams: a reference to a kernel
// parameter handed to a call would copy the whole block to the stack.
__device__ __noinline__ void ion_birth(IonState I, long long cap, double sigma, uint64_t seed,
                                       SimCounters *cnt, uint64_t id, long long step, double r,
                                       double z) {
  const unsigned long long k = atomicAdd(&cnt->n_ions, 1ull);
  if (k >= (unsigned long long)cap) { atomicAdd(&cnt->ion_overflow, 1ull); return; }
  const U2 a = draw2(seed, id, step, 2), b = draw2(seed, id, step, 3);
  double sa, ca, sb, cb;
  sincos(2 * GASATT_PI * a.b, &sa, &ca);
  sincos(2 * GASATT_PI * b.b, &sb, &cb);
  const double ra = sigma * sqrt(-2 * log(a.a)), rb = sigma * sqrt(-2 * log(b.a));
  I.rz[k] = make_double2(r, z);
  I.urt[k] = make_double2(ra * ca, ra * sa);
  I.uz[k] = rb * cb;
  I.id[k] = child_id(id, step);
  I.q[k] = 1;
}

// warp-aggregated append of candidate slots to the collision queue
__device__ __forceinline__ void queue_push(bool want, long long p, unsigned long long *n_cand,
                                           int *queue) {
  const unsigned m = __ballot_sync(0xFFFFFFFFu, want);
  if (!m) return;
  const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(n_cand, (unsigned long long)__popc(m));
  base = __shfl_sync(0xFFFFFFFFu, base, leader);
  if (want) queue[base + __popc(m & ((1u << lane) - 1))] = (int)p;
}

// Commit of a particle pass (parity q), run as its own one-thread kernel after
// the pass: the births of the collision kernel that ran before the pass join
// the committed slots, the queue of the pass is labelled with its step, the
// other queue (consumed by that collision kernel) is emptied, and the step
// advances.  Idempotent: only the first commit after a pass does anything.
// (Done at the end of the pass itself, by its last block, the atomics of 592
// blocks on the counters' cache line slowed the pass by a tenth.)
__device__ __forceinline__ void k_commit_body(SimCounters *cnt, int q) {
  if (!cnt->uncommitted) return;
  const unsigned long long nt = cnt->n_total + cnt->n_births;
  cnt->n_total = nt < cnt->cap ? nt : cnt->cap;
  cnt->n_births = 0;
  cnt->cand_step[q] = cnt->step;
  cnt->n_cand[1 - q] = 0;
  cnt->step += 1;
  cnt->uncommitted = 0;
}
__global__ void k_commit(SimCounters *cnt, int q) { k_commit_body(cnt, q); }

// ------------------------------------------------------ deposit
// Each particle's four node contributions (q FN v w, both components) are
// integers, so every summation order gives the same grid.  The lanes of a warp
// that share a node quad (the sort key; the quad fixes the four node indices)
// are summed with redux.sync, one quad per round, and the first lane of the
// quad adds the eight sums with 64-bit atomics.  Sorted particles put one to
// three quads in a warp; after kDepRounds rounds the lanes left add their own
// contributions.
constexpr int kDepRounds = 4;

// FP64-form contribution, |v| <= 2^48, summed as hi 2^24 + lo with lo in
// [0, 2^24): both 32-lane partial sums fit int32, the recombination is exact
__device__ __forceinline__ long long warp_sum(long long v) {
  const int lo = (int)(v & 0xFFFFFFLL), hi = (int)(v >> 24);
  const long long slo = __reduce_add_sync(0xFFFFFFFFu, lo);
  const long long shi = __reduce_add_sync(0xFFFFFFFFu, hi);
  return shi * (1LL << 24) + slo;
}

template <typename VT>
__device__ __forceinline__ void deposit_atomic(const int64_t a[4], const VT vr[4],
                                               const VT vz[4], unsigned long long *Jr,
                                               unsigned long long *Jz) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (vr[k]) atomicAdd(Jr + a[k], (unsigned long long)(long long)vr[k]);
    if (vz[k]) atomicAdd(Jz + a[k], (unsigned long long)(long long)vz[k]);
  }
}

template <typename VT>
__device__ __forceinline__ void warp_deposit(bool act, unsigned key, const int64_t a[4],
                                             const VT vr[4], const VT vz[4],
                                             unsigned long long *Jr, unsigned long long *Jz) {
  const int lane = threadIdx.x & 31;
  unsigned pending = __ballot_sync(0xFFFFFFFFu, act);
#pragma unroll 1
  for (int round = 0; round < kDepRounds && pending; ++round) {
    const int leader = __ffs(pending) - 1;
    const unsigned lk = __shfl_sync(0xFFFFFFFFu, key, leader);
    const bool mine = act && key == lk;
    pending &= ~__ballot_sync(0xFFFFFFFFu, mine);
    long long sr[4], sz[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      sr[q] = warp_sum(mine ? vr[q] : (VT)0);
      sz[q] = warp_sum(mine ? vz[q] : (VT)0);
    }
    if (lane == leader) deposit_atomic<long long>(a, sr, sz, Jr, Jz);
  }
  if ((pending >> lane) & 1u) deposit_atomic<VT>(a, vr, vz, Jr, Jz);
}


// ----------------------------------------------------------- FP64 form
__device__ __forceinline__ void halfdrift64(double &r, double &z, double &ur, double &ut,
                                            double &uz, bool &alive, const SimParams &P) {
  const double g = sqrt(1 + (ur * ur + ut * ut + uz * uz) / (P.c * P.c));
  const double X = r + 0.5 * (ur / g) * P.dt;
  const double Y = 0.5 * (ut / g) * P.dt;
  double Z = z + 0.5 * (uz / g) * P.dt;
  const double rn = sqrt(X * X + Y * Y);
  const double cs = rn > 0 ? X / rn : 1.0, sn = rn > 0 ? Y / rn : 0.0;
  const double nur = cs * ur + sn * ut, nut = -sn * ur + cs * ut;
  ur = nur; ut = nut;
  if (rn > P.Rp) alive = false;
  if (Z > P.Lp) { Z = 2 * P.Lp - Z; uz = -uz; }
  if (Z < 0) { Z = -Z; uz = -uz; }
  r = rn; z = Z;
}

__device__ __forceinline__ void deposit_values64(const SimParams &P, double r, double z,
                                                 double ur, double ut, double uz, double q,
                                                 int64_t a[4], long long vr[4], long long vz[4],
                                                 unsigned &key) {
  const double g = sqrt(1 + (ur * ur + ut * ut + uz * uz) / (P.c * P.c));
  const double vrr = ur / g, vzz = uz / g;
  double b[4];
  const int ar = em7_weights_ld(r, z, P.nr, P.nz, P.ldj, P.dr, P.dz, a, b);
  const int az = (int)floor(z / P.dz - 0.5);
  key = (unsigned)((ar + 1) + (az + 1) * (P.nr + 1));
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    vr[k] = __double2ll_rn(P.FN * b[k] * q * vrr * P.dep);
    vz[k] = __double2ll_rn(P.FN * b[k] * q * vzz * P.dep);
  }
}

// The particles [beg, end) of the FP64 pass of step `step` (beg a multiple
// of 32 apart from the block's first warp): mode 0: full step - kick, drift
// (two half drifts), deposit; collision candidates go to queue q for k_mcc64;
// mode 1: half drift + deposit only (start of a run); mode 2: kick + half
// drift only, ending at integer time (end of a run).
__device__ __forceinline__ void range64(const SimParams &P, const State64 &S,
                                        const Fields<double> &F, SimCounters *cnt, int *queue,
                                        int mode, int q, long long step, long long beg,
                                        long long end) {
  const int lane = threadIdx.x & 31;
  unsigned lost = 0;
  for (long long base = beg + (threadIdx.x & ~31); base < end; base += blockDim.x) {
    const long long p = base + lane;
    bool act = p < end;
    double2 rz = make_double2(-1.0, 0.0), urt = make_double2(0.0, 0.0);
    double uz = 0;
    if (act) {
      rz = S.rz[p];
      act = rz.x >= 0;
    }
    bool cand = false;
    if (act) {
      urt = S.urt[p]; uz = S.uz[p];
      double r = rz.x, z = rz.y, ur = urt.x, ut = urt.y;
      bool alive = true;
      if (mode != 1) {
        double E_r, E_z, Hp;
        gather3s<double>(F.Er, F.Ez, F.H, P.nr, P.nz, P.ldf, P.ldf, P.ldf, P.dr, P.dz, r, z, E_r,
                         E_z, Hp);
        const double B = P.mu0 * Hp;
        boris(ur, ut, uz, E_r, 0.0, E_z, 0.0, B, 0.0, P.qm_dt2, P.c);
        halfdrift64(r, z, ur, ut, uz, alive, P);
      }
      if (alive && mode != 2) halfdrift64(r, z, ur, ut, uz, alive, P);
      if (alive && mode == 0) cand = null_candidate(P, S.id[p], step);
      if (!alive) {
        lost++;
        r = -1.0;
        count_wall_loss(cnt, (ur * ur + ut * ut + uz * uz) / (P.c * P.c), P.me * P.c * P.c / P.qe);
      }
      rz = make_double2(r, z); urt = make_double2(ur, ut);
      S.rz[p] = rz; S.urt[p] = urt; S.uz[p] = uz;
      act = alive && mode != 2;
    }
    queue_push(cand, p, &cnt->n_cand[q], queue + (long long)q * P.cap);
    int64_t a[4] = {0, 0, 0, 0};
    long long vr[4] = {0, 0, 0, 0}, vz[4] = {0, 0, 0, 0};
    unsigned key = 0;
    if (act) deposit_values64(P, rz.x, rz.y, urt.x, urt.y, uz, -P.qe, a, vr, vz, key);
    warp_deposit<long long>(act, key, a, vr, vz, P.Jr, P.Jz);
  }
  lost = __reduce_add_sync(0xFFFFFFFFu, lost);
  if (lane == 0 && lost) atomicAdd(&cnt->lost, (unsigned long long)lost);
}

__global__ void __launch_bounds__(kBlock, 3) k_pass64(SimParams P, State64 S, Fields<double> F,
                                                      SimCounters *cnt, int *queue, int mode,
                                                      int q) {
  const long long n0 = slots_in_use(cnt);
  const long long step = cnt->step;
  if (blockIdx.x == 0 && threadIdx.x == 0) cnt->uncommitted = 1;
  // each block takes a contiguous chunk of the (cell-sorted) particles, so its
  // field reads stay in a narrow band of grid rows
  const long long chunk = (n0 + gridDim.x - 1) / gridDim.x;
  const long long beg = (long long)blockIdx.x * chunk, end = min(beg + chunk, n0);
  range64(P, S, F, cnt, queue, mode, q, step, beg, end);
}

// The collision of candidate slot p queued at step `step` (FP64 form): MCC,
// the ion and the secondary's birth at the parent's position.  n0: the
// committed slots (births land beyond).
__device__ __forceinline__ void mcc64_one(const SimParams &P, const State64 &S, SimCounters *cnt,
                                          long long p, long long step, long long n0) {
  const double2 rz = S.rz[p], urt = S.urt[p];
  double ur = urt.x, ut = urt.y, uz = S.uz[p];
  const uint64_t id = S.id[p];
  Birth b;
  const double ng = gas_density(P, (int)floor(rz.x / P.dr), (int)floor(rz.y / P.dz));
  const int ev = mcc_event<false>(P, id, step, ur, ut, uz, b, ng);
  count_event(cnt, ev, b);
  if (ev == 2 && P.ion_cap > 0)
    ion_birth(P.ion, P.ion_cap, ion_spread(P, (int)floor(rz.x / P.dr), (int)floor(rz.y / P.dz)),
              P.seed, cnt, id, step, rz.x, rz.y);
  if (b.born) {
    const unsigned long long kb = atomicAdd(&cnt->n_births, 1ull);
    const long long slot = n0 + (long long)kb;
    if (slot < P.cap) {
      S.rz[slot] = rz;
      S.urt[slot] = make_double2(b.ux, b.uy);
      S.uz[slot] = b.uz;
      S.id[slot] = child_id(id, step);
    } else {
      atomicAdd(&cnt->cap_overflow, 1ull);
    }
  }
  S.urt[p] = make_double2(ur, ut); S.uz[p] = uz;
}

// The collisions of the pass that filled queue q, at the end of its step
// (after the drift and the deposit): the MCC changes the velocity, and an
// ionization appends its secondary at the parent's position.  Nothing here
// reads or writes the fields or the current, so it can run beside the next
// field update.
__global__ void __launch_bounds__(kMccBlock) k_mcc64(SimParams P, State64 S, SimCounters *cnt,
                                                     const int *queue, int q) {
  // one candidate per warp (lane 0): the collision branches differ a lot in
  // length, and lanes on different branches would run them one after another
  if ((threadIdx.x & 31) != 0) return;
  const long long n0 = (long long)cnt->n_total;
  const long long step = cnt->cand_step[q];
  const long long nq = (long long)cnt->n_cand[q];
  const int *qu = queue + (long long)q * P.cap;
  const long long nwarps = (long long)gridDim.x * (kMccBlock / 32);
  for (long long k = (blockIdx.x * (long long)kMccBlock + threadIdx.x) >> 5; k < nq; k += nwarps)
    mcc64_one(P, S, cnt, qu[k], step, n0);
}

constexpr int kMaxBatch = 256;               // cells a batch holds at most

// the cell of work item k: the last c with prefix[c] <= k (prefix ascending,
// prefix[0] = 0, n cells)
__device__ __forceinline__ int cell_of_item(const long long *prefix, int n, long long k) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= k) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// ------------------------------------------------------- batched FP64 step
struct BatchCell64 {
  SimParams P[2];             // deposit into current buffer 0 / 1
  State64 S[2];
  SimCounters *cnt;
  int *queue;
  Fields<double> F[2];        // field buffers 0 / 1 (the pass into current buffer jb reads F[jb])
};
constexpr int kChunk64 = 2048;               // particles per work item of the batched FP64 pass

__global__ void k_batch_commit64(const BatchCell64 *__restrict__ cells, int ncell, int q) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x)
    k_commit_body(cells[c].cnt, q);
}

// the collisions queued (parity q) by every cell's last pass, one per warp
__global__ void __launch_bounds__(kMccBlock) k_batch_mcc64(const BatchCell64 *__restrict__ cells,
                                                           int ncell, int cur, int q) {
  __shared__ long long pre[kMaxBatch + 1];
  for (int c = threadIdx.x; c < ncell; c += blockDim.x) pre[c + 1] = (long long)cells[c].cnt->n_cand[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    pre[0] = 0;
    for (int c = 0; c < ncell; ++c) pre[c + 1] += pre[c];
  }
  __syncthreads();
  if ((threadIdx.x & 31) != 0) return;
  const long long nq = pre[ncell];
  const long long nwarps = (long long)gridDim.x * (kMccBlock / 32);
  for (long long k = (blockIdx.x * (long long)kMccBlock + threadIdx.x) >> 5; k < nq; k += nwarps) {
    const int c = cell_of_item(pre, ncell, k);
    const BatchCell64 &C = cells[c];
    SimCounters *cc = C.cnt;
    const int *qu = C.queue + (long long)q * C.P[0].cap;
    mcc64_one(C.P[0], C.S[cur], cc, qu[k - pre[c]], cc->cand_step[q], (long long)cc->n_total);
  }
}

// The FP64 pass of every cell of a batch: (cell, chunk of kChunk64) work
// items from one counter (*chunk_next, zeroed before the launch).
__global__ void __launch_bounds__(kBlock, 3) k_batch_pass64(const BatchCell64 *__restrict__ cells,
                                                            int ncell, int cur, int jb, int mode,
                                                            int q, unsigned long long *chunk_next) {
  __shared__ long long pre[kMaxBatch + 1];
  __shared__ long long item_at;
  for (int c = threadIdx.x; c < ncell; c += blockDim.x)
    pre[c + 1] = (slots_in_use(cells[c].cnt) + kChunk64 - 1) / kChunk64;
  __syncthreads();
  if (threadIdx.x == 0) {
    pre[0] = 0;
    for (int c = 0; c < ncell; ++c) pre[c + 1] += pre[c];
    if (blockIdx.x == 0)
      for (int c = 0; c < ncell; ++c) cells[c].cnt->uncommitted = 1;
  }
  __syncthreads();
  const long long nitem = pre[ncell];
  for (;;) {
    if (threadIdx.x == 0) item_at = (long long)atomicAdd(chunk_next, 1ull);
    __syncthreads();
    const long long g = item_at;
    __syncthreads();
    if (g >= nitem) break;
    const int c = cell_of_item(pre, ncell, g);
    const BatchCell64 &C = cells[c];
    SimCounters *cc = C.cnt;
    const long long n0 = slots_in_use(cc);
    const long long beg = (g - pre[c]) * kChunk64, end = min(beg + kChunk64, n0);
    range64(C.P[jb], C.S[cur], C.F[jb], cc, C.queue, mode, q, cc->step, beg, end);
  }
}

// ----------------------------------------------------------- ions
// Before each push the ions are sorted by deposit node quad (the electrons'
// sort key) from the store into a scratch store, dropping the dead; the push
// reads the scratch and writes the store back in that order.  Ions hardly
// move between pushes, so only those born since the last push are out of
// place, and the lanes of a warp then share their deposit nodes (the warp
// sums replace most of the atomics on the crowded cells near the axis).
__device__ __forceinline__ int ion_cell(const IonState &I, long long p, int nr, int nz, double dr,
                                        double dz) {
  const double2 rz = I.rz[p];
  if (rz.x < 0) return -1;
  int ar = (int)floor(rz.x / dr - 0.5) + 1, az = (int)floor(rz.y / dz - 0.5) + 1;
  ar = min(max(ar, 0), nr);
  az = min(max(az, 0), nz);
  return ar + az * (nr + 1);
}

__device__ __forceinline__ long long ions_in_use(const SimCounters *cnt, long long cap) {
  const unsigned long long nc = cnt->n_ions;
  return (long long)(nc < (unsigned long long)cap ? nc : cap);
}

__global__ void k_ion_hist(IonState I, const SimCounters *cnt, long long cap, int nr, int nz,
                           double dr, double dz, int *count) {
  const long long n = ions_in_use(cnt, cap);
  for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n;
       base += (long long)gridDim.x * blockDim.x) {
    const long long p = base + (threadIdx.x & 31);
    const int c = p < n ? ion_cell(I, p, nr, nz, dr, dz) : -1;
    const unsigned live = __ballot_sync(0xFFFFFFFFu, c >= 0);
    if (c < 0) continue;
    const unsigned mask = __match_any_sync(live, c);
    if ((__ffs(mask) - 1) == (int)(threadIdx.x & 31)) atomicAdd(count + c, __popc(mask));
  }
}

__global__ void k_ion_scatter(IonState A, IonState B, const SimCounters *cnt, long long cap,
                              int nr, int nz, double dr, double dz, const int *offset,
                              int *cursor) {
  const long long n = ions_in_use(cnt, cap);
  const int lane = threadIdx.x & 31;
  for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n;
       base += (long long)gridDim.x * blockDim.x) {
    const long long p = base + lane;
    const int c = p < n ? ion_cell(A, p, nr, nz, dr, dz) : -1;
    const unsigned live = __ballot_sync(0xFFFFFFFFu, c >= 0);
    if (c < 0) continue;
    const unsigned mask = __match_any_sync(live, c);
    const int leader = __ffs(mask) - 1;
    int basepos = 0;
    if (lane == leader) basepos = atomicAdd(cursor + c, __popc(mask));
    basepos = __shfl_sync(mask, basepos, leader);
    const long long dst = (long long)offset[c] + basepos + __popc(mask & ((1u << lane) - 1));
    B.rz[dst] = A.rz[p]; B.urt[dst] = A.urt[p]; B.uz[dst] = A.uz[p];
    B.id[dst] = A.id[p]; B.q[dst] = A.q[p];
  }
}

// the live ions are now the first offset[nbin] slots
__global__ void k_ion_sort_finish(SimCounters *cnt, const int *offset, int nbin) {
  cnt->n_ions = (unsigned long long)offset[nbin];
}

// Ion push, once every ion_subcycle electron steps: P is the simulation's
// parameter block with dt = the ion step, qm_dt2 = q_e/m_ion dt/2 and the
// ion current buffers as Jr/Jz (cleared before the launch), dep = the
// fixed-point factor of the ion current.  Per ion of the sorted scratch
// store src: gather, Boris kick with charge Z q_e, two half drifts (the
// electrons' walls: absorbed beyond Rp, reflected at z = 0 and Lp), deposit
// of Z q_e FN v at the new position; the ion goes back to the store P.ion at
// the same index.  The field update adds the ion current to the electrons'
// until the next push (charge moved over the ion step = the held current x
// the ion step).
template <typename T>
__global__ void __launch_bounds__(kBlock) k_ion_push(SimParams P, Fields<T> F, SimCounters *cnt,
                                                     IonState src) {
  const long long n = ions_in_use(cnt, P.ion_cap);
  const IonState I = P.ion;
  unsigned lost = 0;
  for (long long base = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); base < n;
       base += (long long)gridDim.x * blockDim.x) {
    const long long p = base + (threadIdx.x & 31);
    bool act = p < n;
    double2 rz = make_double2(-1.0, 0.0), urt = make_double2(0.0, 0.0);
    double uz = 0, Zq = 0;
    if (act) {
      rz = src.rz[p];
      act = rz.x >= 0;
    }
    if (act) {
      urt = src.urt[p]; uz = src.uz[p];
      const int8_t q = src.q[p];
      Zq = (double)q;
      I.id[p] = src.id[p]; I.q[p] = q;
      double r = rz.x, z = rz.y, ur = urt.x, ut = urt.y;
      bool alive = true;
      double E_r, E_z, Hp;
      gather3s<T>(F.Er, F.Ez, F.H, P.nr, P.nz, P.ldf, P.ldf, P.ldf, P.dr, P.dz, r, z, E_r, E_z, Hp);
      boris(ur, ut, uz, E_r, 0.0, E_z, 0.0, P.mu0 * Hp, 0.0, Zq * P.qm_dt2, P.c);
      halfdrift64(r, z, ur, ut, uz, alive, P);
      if (alive) halfdrift64(r, z, ur, ut, uz, alive, P);
      if (!alive) {
        lost++;
        r = -1.0;
        count_wall_loss(cnt, (ur * ur + ut * ut + uz * uz) / (P.c * P.c), P.m_ion * P.c * P.c / P.qe);
      }
      rz = make_double2(r, z); urt = make_double2(ur, ut);
      I.rz[p] = rz; I.urt[p] = urt; I.uz[p] = uz;
      act = alive;
    }
    int64_t a[4] = {0, 0, 0, 0};
    long long vr[4] = {0, 0, 0, 0}, vz[4] = {0, 0, 0, 0};
    unsigned key = 0;
    if (act) deposit_values64(P, rz.x, rz.y, urt.x, urt.y, uz, Zq * P.qe, a, vr, vz, key);
    warp_deposit<long long>(act, key, a, vr, vz, P.Jr, P.Jz);
  }
  lost = __reduce_add_sync(0xFFFFFFFFu, lost);
  if ((threadIdx.x & 31) == 0 && lost) atomicAdd(&cnt->ion_lost, (unsigned long long)lost);
}

// ion diagnostics: alive, sum of charge numbers, kinetic energy (fixed point)
__global__ void k_ion_diag(IonState I, long long cap, SimCounters *cnt, double c, double m_ion,
                           double qe) {
  const unsigned long long nc = cnt->n_ions;
  const long long n = (long long)(nc < (unsigned long long)cap ? nc : cap);
  unsigned long long kin = 0, alive = 0, charge = 0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    if (I.rz[p].x < 0) continue;
    const double2 a = I.urt[p];
    const double w = I.uz[p];
    const double u2 = (a.x * a.x + a.y * a.y + w * w) / (c * c);
    const double g = sqrt(1 + u2);
    kin += (unsigned long long)__double2ll_rn(m_ion * c * c * (u2 / (g + 1)) / qe * 4294967296.0);
    alive++;
    charge += (unsigned long long)I.q[p];
  }
  for (int o = 16; o; o >>= 1) {
    kin += __shfl_down_sync(0xFFFFFFFFu, kin, o);
    alive += __shfl_down_sync(0xFFFFFFFFu, alive, o);
    charge += __shfl_down_sync(0xFFFFFFFFu, charge, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&cnt->ion_kin_fx, kin);
    atomicAdd(&cnt->ion_alive, alive);
    atomicAdd(&cnt->ion_charge, charge);
  }
}

__global__ void k_ion_load(IonState I, const double *r, const double *z, const double *ur,
                           const double *ut, const double *uz, const uint64_t *id,
                           const int8_t *q, long long n) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    I.rz[p] = make_double2(r[p], z[p]);
    I.urt[p] = make_double2(ur[p], ut[p]);
    I.uz[p] = uz[p];
    I.id[p] = id[p];
    I.q[p] = q ? q[p] : (int8_t)1;
  }
}

__global__ void k_ion_read(IonState I, double *r, double *z, double *ur, double *ut, double *uz,
                           uint64_t *id, int8_t *q, long long n) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    const double2 a = I.rz[p], b = I.urt[p];
    r[p] = a.x; z[p] = a.y; ur[p] = b.x; ut[p] = b.y; uz[p] = I.uz[p];
    id[p] = I.id[p];
    q[p] = I.q[p];
  }
}

// ----------------------------------------------------------- FP32 form
// 1/sqrt(x) refined by one Newton step: the hardware estimate is biased, and
// a biased rotation normaliser or gamma makes the FP32 energy drift steadily
__device__ __forceinline__ float rsqrt_nr(float x) {
  const float y = rsqrtf(x);
  return y * fmaf(-0.5f * x * y, y, 1.5f);
}

// Packed pairs: Blackwell issues two FP32 operations of a float2 as one
// instruction (__fadd2/__fmul2/__ffma2, sm_100); the FP32 push pairs its
// independent r/z (or column/row) operations this way.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// a + d with stochastic rounding.  The per-step velocity changes of the FP32
// form (a drift rotation by a small angle, a kick in a weak field) are often
// below one float ulp of u; rounding them to nearest would bias |u| steadily.
// With h the spacing of the floats in a's binade and U uniform in [0, 1), the
// sum a + d + sign(a) U h rounded toward zero is a + d rounded to one of its
// two neighbours on that grid, the far one with probability equal to the
// distance from the near one in units of h: unbiased as long as a + d stays
// in a's binade (within |d| of a power of two the grid changes and the split
// is off by up to a factor 2; there |d| << |a| makes that a rare, tiny
// error).  a + d + U h is formed exactly enough in one FMA (d and U h are
// both small against a) and rounded once.  U = (k + 1/2) 2^-16, k a 16-bit
// random number, is built as a float in [1, 2) minus 1; a = 0 gives h = 0
// and the exact d.  Done on a pair of components: k from the low 16 bits of r
// for x, from the high 16 for y.
__device__ __forceinline__ float2 sround_add2(float2 a, float2 d, uint32_t r) {
  const float2 h = __fmul2_rn(f2(__int_as_float(__float_as_int(a.x) & 0x7F800000),
                                 __int_as_float(__float_as_int(a.y) & 0x7F800000)),
                              f2(1.1920928955078125e-07f));
  const float2 u = __fadd2_rn(f2(__uint_as_float(0x3F800040u | ((r & 0xFFFFu) << 7)),
                                 __uint_as_float(0x3F800040u | ((r >> 16) << 7))),
                              f2(-1.0f));
  return __fadd2_rz(a, __ffma2_rn(f2(copysignf(u.x, a.x), copysignf(u.y, a.y)), h, d));
}

// Floors and nearest integers in FP32 without conversions: for |x| < 2^22,
// x + 1.5 2^23 lies where the floats are one apart, so rounding that sum
// down (or to nearest) gives 1.5 2^23 + floor(x) (or + rint(x)) exactly and
// its bit pattern minus 0x4B400000 is the integer.

// half-cell staggered index/weight: position ic + f measured from node ic-1/2
__device__ __forceinline__ void half_shift(int ic, float f, int &a, float &w) {
  const bool up = f >= 0.5f;
  a = up ? ic : ic - 1;
  w = up ? f - 0.5f : f + 0.5f;
}

// specular reflection of the cell coordinate (iz, fz) into [0, nz)
__device__ __forceinline__ void reflect_z(int &iz, float &fz, float &uz, int nz) {
  if (iz < 0 || iz >= nz) {
    iz = iz < 0 ? -iz - 1 : 2 * nz - iz - 1;
    fz = 1.f - fz;
    uz = -uz;
    if (fz >= 1.f) { fz = 0.f; iz += 1; }
    if (iz > nz - 1) { iz = nz - 1; fz = 0.99999994f; }
    if (iz < 0) { iz = 0; fz = 0.f; }
  }
}

// Straight-line drift in cell units over (hr, hz) cells per unit beta:
// (P.hdr, P.hdz) is a half step, twice that a full step.  Two half drifts at
// the same velocity are one full drift: the Cartesian path is the same line,
// the radius along a line is convex (a particle inside the wall at both ends
// is inside at the midpoint), and the end reflection is specular.  The new
// radius comes from the exact difference r' - rc = (dx (2 rc + dx) + dy^2) /
// (r' + rc) (no cancellation at large rc); (u_r, u_theta) turn by the drift
// angle a, written with the small quantities sin a and 1 - cos a = sin^2 a /
// (1 + cos a) and added to u with stochastic rounding (rb: two 16-bit random
// numbers).
__device__ __forceinline__ void drift32(int &ir, int &iz, float &fr, float &fz, float &ur,
                                        float &ut, float &uz, bool &alive, const SimParams &P,
                                        uint32_t rb, float hr, float hz, float &ig) {
  // 1/gamma, kept by the turn.  (The hardware estimate is enough here: it only
  // scales the displacement and the current, and the turn keeps |u| whatever
  // it is; the kick's 1/gamma is refined.)
  ig = rsqrtf(fmaf(ur, ur, fmaf(ut, ut, fmaf(uz, uz, 1.0f))));
  const float2 dxy = __fmul2_rn(__fmul2_rn(f2(ur, ut), f2(ig)), f2(hr));   // (dx, dy)
  const float dx = dxy.x, dy = dxy.y, dzz = uz * ig * hz;
  const float rc = (float)ir + fr;
  const float X = rc + dx;
  const float r2 = fmaf(X, X, dy * dy);
  // (products that feed a sum are __fmul_rn: never contracted into an FMA,
  // so every kernel that inlines this rounds the same way)
  const float irn = rsqrt_nr(r2);                    // 1/r' (inf at r' = 0)
  const float rn = __fmul_rn(r2, irn);
  const float sn = r2 > 0.f ? dy * irn : 0.f;
  const float s2 = __fmul_rn(sn, sn);
  const float cs = r2 > 0.f ? X * irn : 1.f;         // cos a
  const float c1 = X >= 0.f ? __fdividef(s2, 1.f + cs) : 1.f - cs;   // 1 - cos a
  // (du_r, du_theta) = (sn ut - c1 ur, -sn ur - c1 ut)
  const float2 du = __ffma2_rn(f2(sn, -sn), f2(ut, ur), __fmul2_rn(f2(ur, ut), f2(-c1)));
  const float2 u2 = sround_add2(f2(ur, ut), du, rb);
  ur = u2.x;
  ut = u2.y;
  const float den = rn + rc;
  const float drr = den > 0.f ? __fdividef(fmaf(dx, 2.f * rc + dx, dy * dy), den) : 0.f;
  // floor of both offsets at once (take_floor on a pair)
  const float2 f = __fadd2_rn(f2(fr, fz), f2(drr, dzz));
  const float2 t = __fadd2_rd(f, f2(12582912.0f));
  const float2 g = __fadd2_rn(f, neg2(__fadd2_rn(t, f2(-12582912.0f))));
  fr = g.x;
  fz = g.y;
  ir += __float_as_int(t.x) - 0x4B400000;
  iz += __float_as_int(t.y) - 0x4B400000;
  if (ir < 0) { ir = 0; fr = 0.f; }
  alive = alive && ir < P.nr;
  reflect_z(iz, fz, uz, P.nz);
}

// The four deposit nodes (columns ca, cb; rows ra, rb; clamped one-sided at
// the edges as EM7.cu:56-202) and the fixed-point contributions.  perm (0..3)
// permutes the node order: bit 0 swaps the columns, bit 1 the rows, so the
// order is (c0,r0), (c1,r0), (c0,r1), (c1,r1) with (c0, c1) = (ca, cb) or
// (cb, ca) and likewise rows; each node's integer is the same whatever the
// order (its weight is the same product of the same two factors).  The
// weights sum to 1, so one particle adds at most 2^20 in magnitude to any
// node, even where clamped nodes merge.  ig: 1/gamma of u (the drift's,
// which turns u without changing |u|).
__device__ __forceinline__ void deposit_nodes32(const SimParams &P, int ir, int iz, float fr,
                                                float fz, float ur, float uz, float ig, int perm,
                                                int &c0, int &c1, int &r0, int &r1, int vr[4],
                                                int vz[4]) {
  int ar, az;
  float wr, wz;
  half_shift(ir, fr, ar, wr);
  half_shift(iz, fz, az, wz);
  const int ca = max(ar, 0), cb = min(ar + 1, P.nr - 1);
  const int ra = max(az, 0), rb = min(az + 1, P.nz - 1);
  const bool sc = perm & 1, sr = perm & 2;
  c0 = sc ? cb : ca; c1 = sc ? ca : cb;
  r0 = sr ? rb : ra; r1 = sr ? ra : rb;
  const float2 om = __fadd2_rn(f2(1.f), f2(-wr, -wz));        // (1 - wr, 1 - wz)
  const float2 A = sc ? f2(wr, om.x) : f2(om.x, wr);         // column factors of c0, c1
  const float B0 = sr ? wz : om.y, B1 = sr ? om.y : wz;       // row factors of r0, r1
  const float2 w01 = __fmul2_rn(A, f2(B0)), w23 = __fmul2_rn(A, f2(B1));
  const float2 k = __fmul2_rn(__fmul2_rn(f2(P.depf), f2(ur, uz)), f2(ig));   // (kr, kz)
  const float2 C = f2(12582912.0f);
  const float2 v0 = __ffma2_rn(k, f2(w01.x), C), v1 = __ffma2_rn(k, f2(w01.y), C);
  const float2 v2 = __ffma2_rn(k, f2(w23.x), C), v3 = __ffma2_rn(k, f2(w23.y), C);
  vr[0] = __float_as_int(v0.x) - 0x4B400000; vz[0] = __float_as_int(v0.y) - 0x4B400000;
  vr[1] = __float_as_int(v1.x) - 0x4B400000; vz[1] = __float_as_int(v1.y) - 0x4B400000;
  vr[2] = __float_as_int(v2.x) - 0x4B400000; vz[2] = __float_as_int(v2.y) - 0x4B400000;
  vr[3] = __float_as_int(v3.x) - 0x4B400000; vz[3] = __float_as_int(v3.y) - 0x4B400000;
}

// FP32-form deposit window: int32 sums of one chunk of particles on the grid
// rows [row0, row0 + rows) in shared memory.  A chunk holds at most kChunkMax
// particles, so a node's window sum stays below kChunkMax * 2^20 < 2^31.  A
// node's two sums (r, z) are adjacent words, so one address serves both
// atomics; rows are ws >= nr nodes apart with ws = 3 (mod 32), so the 3 x 3
// nodes around a warp's particles sit in 9 different bank pairs.  Nodes
// outside the window go straight to the grid with 64-bit atomics; the window
// is added to the grid with one 64-bit atomic per touched node.
constexpr int kWinNodes = 4096;           // nodes (two int32 sums each)
constexpr int kChunkMax = 7 * kBlock;     // 1792 particles (the default chunk)

struct Win32 {
  int *rz;                  // node k: r at rz[2k], z at rz[2k + 1]
  int row0, rows, ws;
};

__host__ __device__ inline int win_stride(int nr) { return nr + ((3 - nr % 32) + 32) % 32; }

__device__ __forceinline__ void win_node(const Win32 &w, const SimParams &P, int col, int row,
                                         int vr, int vz) {
  const unsigned lr = (unsigned)(row - w.row0);
  if (lr < (unsigned)w.rows) {
    const int k = (int)lr * w.ws + col;
    atomicAdd(w.rz + 2 * k, vr);
    atomicAdd(w.rz + 2 * k + 1, vz);
  } else {
    const int64_t g = col + (int64_t)row * P.ldj;
    if (vr) atomicAdd(P.Jr + g, (unsigned long long)(long long)vr);
    if (vz) atomicAdd(P.Jz + g, (unsigned long long)(long long)vz);
  }
}

// FP32 state flags.  The in-cell offsets fr, fz are >= 0, so their sign bits
// are free: the sign of fr marks a pending collision (the particle sits in the
// collision queue of the pass that pushed it last), the sign of fz is the
// parity of the step in which the particle was pushed last.
constexpr uint32_t kSign = 0x80000000u;

__device__ __forceinline__ uint4 pack32(int ir, int iz, float fr, float fz, float ur, bool alive,
                                        bool pending = false, int par = 0) {
  return make_uint4(alive ? (((uint32_t)iz << 16) | (uint32_t)ir) : kDead,
                    __float_as_uint(fr) | (pending ? kSign : 0u),
                    __float_as_uint(fz) | (par ? kSign : 0u), __float_as_uint(ur));
}

// One particle's push in step `step`.  mode 0: gather, Boris kick, drift of
// the whole step, null-collision candidate test; mode 1: half drift (start of
// a run); mode 2: gather, kick, half drift to integer time (end of a run).
// Returns whether the particle is a collision candidate (alive, mode 0).
template <int MODE>
__device__ __forceinline__ bool push32(const SimParams &P, const Fields<float> &F, uint64_t id,
                                       long long step, int &ir, int &iz, float &fr,
                                       float &fz, float &ur, float &ut, float &uz, bool &alive,
                                       float &ig) {
  // block 0 of this particle's stream: words 0-1 decide the null-collision
  // candidate, words 2-3 drive the stochastic rounding of the kick and the turn
  uint32_t c[4] = {(uint32_t)id, (uint32_t)(id >> 32), (uint32_t)step, 0u};
  if (MODE == 1) {
    philox4x32_10(c, P.pk);
    drift32(ir, iz, fr, fz, ur, ut, uz, alive, P, c[3], P.hdr, P.hdz, ig);
    return false;
  }
  int ar, az;
  float wr, wz;
  half_shift(ir, fr, ar, wr);
  half_shift(iz, fz, az, wz);
  // the field loads go out first, their latency hidden behind Philox: one
  // packed quad per field (corners already clamped at the edges), or the
  // same four corners from the fields themselves (the same floats)
  float4 a4, b4, c4;
  if (P.qEr) {
    a4 = __ldg(P.qEr + ((ar + 1) + iz * (P.nr + 1)));
    b4 = __ldg(P.qEz + (ir + (az + 1) * P.nr));
    c4 = __ldg(P.qH + ((ar + 1) + (az + 1) * (P.nr + 1)));
  } else {
    const int c0 = max(ar, 0), c1 = min(ar + 1, P.nr - 1);
    const int ra = max(az, 0), rb = min(az + 1, P.nz - 1);
    const float *e0 = F.Er + iz * P.ldf, *e1 = e0 + P.ldf;
    a4 = make_float4(__ldg(e0 + c0), __ldg(e0 + c1), __ldg(e1 + c0), __ldg(e1 + c1));
    const float *z0 = F.Ez + ra * P.ldf + ir, *z1 = F.Ez + rb * P.ldf + ir;
    b4 = make_float4(__ldg(z0), __ldg(z0 + 1), __ldg(z1), __ldg(z1 + 1));
    const float *h0 = F.H + ra * P.ldf, *h1 = F.H + rb * P.ldf;
    c4 = make_float4(__ldg(h0 + c0), __ldg(h0 + c1), __ldg(h1 + c0), __ldg(h1 + c1));
  }
  philox4x32_10(c, P.pk);
  // bilinear mixes from the quads' corners (c0,r0), (c1,r0), (c0,r1), (c1,r1)
  // = (x, y, z, w), paired: the low and high rows of each quad along its
  // columns, then Er and Ez along their rows
  const float2 cE = __ffma2_rn(f2(wr), __fadd2_rn(f2(a4.y, a4.w), f2(-a4.x, -a4.z)), f2(a4.x, a4.z));
  const float2 cZ = __ffma2_rn(f2(fr), __fadd2_rn(f2(b4.y, b4.w), f2(-b4.x, -b4.z)), f2(b4.x, b4.z));
  const float2 cH = __ffma2_rn(f2(wr), __fadd2_rn(f2(c4.y, c4.w), f2(-c4.x, -c4.z)), f2(c4.x, c4.z));
  const float2 E = __ffma2_rn(f2(fz, wz), __fadd2_rn(f2(cE.y, cZ.y), f2(-cE.x, -cZ.x)), f2(cE.x, cZ.x));
  const float H = fmaf(wz, cH.y - cH.x, cH.x);
  // Boris in gamma*beta units: E = (Er, 0, Ez), B = (0, mu0 H, 0); the
  // increment u+ - u is formed first, then added with stochastic rounding
  // (random bits: Philox words 2 and 3)
  const float2 he = __fmul2_rn(f2(P.aE), E);                  // (her, hez)
  const float2 um = __fadd2_rn(f2(ur, uz), he);               // (umr, umz)
  const float igm = rsqrt_nr(fmaf(um.x, um.x, fmaf(ut, ut, fmaf(um.y, um.y, 1.0f))));
  const float t = P.aB * H * igm;
  const float s = __fdividef(2.f * t, fmaf(t, t, 1.f));
  const float2 up = __ffma2_rn(f2(-um.y, um.x), f2(t), um);   // (upr, upz)
  const float2 du = __ffma2_rn(f2(-up.y, up.x), f2(s), __fadd2_rn(he, he));
  const float2 uk = sround_add2(f2(ur, uz), du, c[2]);
  ur = uk.x;
  uz = uk.y;
  const float h = MODE == 0 ? 2.f : 1.f;
  drift32(ir, iz, fr, fz, ur, ut, uz, alive, P, c[3], h * P.hdr, h * P.hdz, ig);
  return alive && MODE == 0 && (((((uint64_t)c[0]) << 32) | c[1]) >> 12) < P.cand_below;
}

// ig: the drift's 1/gamma, as in the chunk loop, so that a particle deposits
// the same integers whichever path pushed it
__device__ __forceinline__ void deposit_global32(const SimParams &P, int ir, int iz, float fr,
                                                 float fz, float ur, float uz, float ig) {
  int ca, cb, ra, rb, vr[4], vz[4];
  deposit_nodes32(P, ir, iz, fr, fz, ur, uz, ig, 0, ca, cb, ra, rb, vr, vz);
  const int64_t a[4] = {ca + (int64_t)ra * P.ldj, cb + (int64_t)ra * P.ldj,
                        ca + (int64_t)rb * P.ldj, cb + (int64_t)rb * P.ldj};
  deposit_atomic<int>(a, vr, vz, P.Jr, P.Jz);
}

__device__ __forceinline__ void queue_one(SimCounters *cnt, int *queue, const SimParams &P,
                                          int par, long long p) {
  const unsigned long long k = atomicAdd(&cnt->n_cand[par], 1ull);
  queue[(long long)par * P.cap + (long long)k] = (int)p;
}

// A collision candidate of the previous step (FP32 form), taken by one lane:
// the MCC at the end of step `step` - 1 (FP64 test, branch, energy sharing;
// float turn), the secondary's birth at the parent's position, then the push
// of step `step` for both (push == true) with their current deposited by
// global atomics and their own candidate test, or (push == false) nothing
// more.  The chunk loop of the pass skips these particles (pending flag set,
// or pushed-parity = this step's).
// P: the launch's parameters in global memory (a reference to the kernel's
// own parameter block would make every thread copy it to its stack).
__device__ __noinline__ void candidate32(const SimParams *__restrict__ Pg, Fields<float> F,
                                         State32 S, SimCounters *cnt, int *queue, long long p,
                                         long long step, int mode, bool push, long long n0,
                                         unsigned &lost) {
  const SimParams &P = *Pg;
  const int par = (int)(step & 1);
  const long long cstep = push ? step - 1 : step;      // step whose collision this is
  const uint4 A = S.a[p];
  const float2 B = S.b[p];
  const uint64_t id = S.id[p];
  int ir = (int)(A.x & 0xFFFFu), iz = (int)(A.x >> 16);
  float fr = __uint_as_float(A.y & ~kSign), fz = __uint_as_float(A.z & ~kSign);
  double dux = (double)__uint_as_float(A.w) * P.c, duy = (double)B.x * P.c, duz = (double)B.y * P.c;
  Birth b;
  const int ev = mcc_event<true>(P, id, cstep, dux, duy, duz, b, gas_density(P, ir, iz));
  count_event(cnt, ev, b);
  if (ev == 2 && P.ion_cap > 0)
    ion_birth(P.ion, P.ion_cap, ion_spread(P, ir, iz), P.seed, cnt, id, cstep, ((double)ir + (double)fr) * P.dr,
              ((double)iz + (double)fz) * P.dz);
  const int mark = push ? par : (int)(cstep & 1);
  if (b.born) {
    const unsigned long long kb = atomicAdd(&cnt->n_births, 1ull);
    const long long slot = n0 + (long long)kb;
    if (slot < P.cap) {
      int cir = ir, ciz = iz;
      float cfr = fr, cfz = fz;
      float cur = (float)(b.ux / P.c), cut = (float)(b.uy / P.c), cuz = (float)(b.uz / P.c);
      bool calive = true, cc = false;
      const uint64_t cid = child_id(id, cstep);
      if (push) {
        float cig;
        cc = mode == 0 ? push32<0>(P, F, cid, step, cir, ciz, cfr, cfz, cur, cut, cuz, calive, cig)
           : mode == 1 ? push32<1>(P, F, cid, step, cir, ciz, cfr, cfz, cur, cut, cuz, calive, cig)
                       : push32<2>(P, F, cid, step, cir, ciz, cfr, cfz, cur, cut, cuz, calive, cig);
        if (calive && mode != 2) deposit_global32(P, cir, ciz, cfr, cfz, cur, cuz, cig);
        if (!calive) {
          lost++;
          count_wall_loss(cnt, (double)cur * cur + (double)cut * cut + (double)cuz * cuz, P.me * P.c * P.c / P.qe);
        }
        if (cc) queue_one(cnt, queue, P, par, slot);
      }
      S.a[slot] = pack32(cir, ciz, cfr, cfz, cur, calive, cc, mark);
      S.b[slot] = make_float2(cut, cuz);
      S.id[slot] = cid;
    } else {
      atomicAdd(&cnt->cap_overflow, 1ull);
    }
  }
  float ur = (float)(dux / P.c), ut = (float)(duy / P.c), uz = (float)(duz / P.c);
  bool alive = true, pc = false;
  if (push) {
    float pig;
    pc = mode == 0 ? push32<0>(P, F, id, step, ir, iz, fr, fz, ur, ut, uz, alive, pig)
       : mode == 1 ? push32<1>(P, F, id, step, ir, iz, fr, fz, ur, ut, uz, alive, pig)
                   : push32<2>(P, F, id, step, ir, iz, fr, fz, ur, ut, uz, alive, pig);
    if (alive && mode != 2) deposit_global32(P, ir, iz, fr, fz, ur, uz, pig);
    if (!alive) {
      lost++;
      count_wall_loss(cnt, (double)ur * ur + (double)ut * ut + (double)uz * uz, P.me * P.c * P.c / P.qe);
    }
    if (pc) queue_one(cnt, queue, P, par, p);
  }
  S.a[p] = pack32(ir, iz, fr, fz, ur, alive, pc, mark);
  S.b[p] = make_float2(ut, uz);
}

// Window rows of chunk ch (particles [ch chunk, min(ch chunk + chunk, n0))):
// the node rows of its first and last particles, with a margin for the drift
// since the last sort.  maxrows: rows the window holds for this grid.
__device__ __forceinline__ void chunk_rows32(const SimParams &P, const State32 &S, long long n0,
                                             int chunk, long long ch, int maxrows, int &row0,
                                             int &rows) {
  const long long beg = ch * chunk, end = min(beg + chunk, n0);
  const uint32_t k0 = reinterpret_cast<const uint32_t *>(S.a + beg)[0];
  const uint32_t k1 = reinterpret_cast<const uint32_t *>(S.a + end - 1)[0];
  int lo = P.nz, hi = -1;
  if (k0 != kDead) { lo = min(lo, (int)(k0 >> 16)); hi = max(hi, (int)(k0 >> 16)); }
  if (k1 != kDead) { lo = min(lo, (int)(k1 >> 16)); hi = max(hi, (int)(k1 >> 16)); }
  row0 = 0; rows = maxrows;
  if (hi >= 0) {
    // the chunk's own deposit rows lo-1 .. hi+1 first, then up to three
    // rows either side for the drift since the last sort (a wide grid
    // leaves room for few rows)
    const int core = hi - lo + 3;
    const int below = maxrows >= core + 6 ? 3 : max(1, 1 + (maxrows - core) / 2);
    row0 = min(max(0, lo - below), P.nz - maxrows);
    rows = min(maxrows, hi + 4 - row0);
  }
}

// Bring the state of particles [beg, end) into L2 ahead of their chunk (one
// thread; cp.async.bulk.prefetch.L2, a hint that completes on its own).  beg
// is a multiple of the chunk size, hence even, so every range starts on a
// 16-byte boundary; the sizes are rounded down to 16 bytes.
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
  if (bytes) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
__device__ __forceinline__ void prefetch_chunk32(const State32 &S, long long beg, long long end) {
  const long long n = end - beg;
  if (n <= 0) return;
  prefetch_l2(S.a + beg, (uint32_t)(n * 16));
  prefetch_l2(S.b + beg, (uint32_t)((n * 8) & ~15ll));
  prefetch_l2(S.id + beg, (uint32_t)((n * 8) & ~15ll));
}

// The particles [beg, end) of one chunk of the FP32 pass of step `step`:
// push (push32), collision candidates queued, deposit into the window w
// (nodes outside the window straight to the grid).  The highest window column touched is merged
// into *box_cmax; electrons absorbed at the wall are counted into cnt.
template <int MODE>
__device__ __forceinline__ void chunk32(const SimParams &P, const State32 &S, const Fields<float> &F,
                                        SimCounters *cnt, int *queue, long long step,
                                        int beg, int end, const Win32 &w, int *box_cmax) {
  const int par = (int)(step & 1);
  const uint32_t parbit = par ? kSign : 0u;
  const int lane = threadIdx.x & 31;
  unsigned lost = 0;
  int wc_max = -1;                 // highest window column this lane touched
  // the next iteration's particle is loaded one iteration ahead, so its
  // HBM latency overlaps the current particle's arithmetic
  int base = beg + (int)(threadIdx.x & ~31);
  uint4 An = make_uint4(kDead, 0, 0, 0);
  float2 Bn = make_float2(0.f, 0.f);
  uint64_t idn = 0;
  if (base + lane < end) { An = S.a[base + lane]; Bn = S.b[base + lane]; idn = S.id[base + lane]; }
  for (; base < end; base += kBlock) {
    const int p = base + lane;
    uint4 A = An;
    const float2 B = Bn;
    const uint64_t id = idn;
    {
      const int pn = p + kBlock;
      An = make_uint4(kDead, 0, 0, 0);
      if (pn < end) { An = S.a[pn]; Bn = S.b[pn]; idn = S.id[pn]; }
    }
    // skip the dead, the pending collisions and those already pushed in
    // this step (the candidates the pass has taken)
    bool act = p < end && A.x != kDead && !(A.y & kSign) && (A.z & kSign) != parbit;
    int ir = (int)(A.x & 0xFFFFu), iz = (int)(A.x >> 16);
    float fr = __uint_as_float(A.y & ~kSign), fz = __uint_as_float(A.z & ~kSign);
    float ur = __uint_as_float(A.w), ut = B.x, uz = B.y, ig = 1.f;
    bool cand = false;
    if (act) {
      bool alive = true;
      cand = push32<MODE>(P, F, id, step, ir, iz, fr, fz, ur, ut, uz, alive, ig);
      if (!alive) {
        lost++;
        count_wall_loss(cnt, (double)ur * ur + (double)ut * ut + (double)uz * uz, P.me * P.c * P.c / P.qe);
      }
      S.a[p] = pack32(ir, iz, fr, fz, ur, alive, cand, par);
      S.b[p] = make_float2(ut, uz);
      act = alive && MODE != 2;
    }
    queue_push(cand, p, &cnt->n_cand[par], queue + (long long)par * P.cap);
    // Deposit: each lane adds its own eight contributions to the window,
    // visiting its four nodes in an order permuted by lane & 3 (columns
    // swapped on bit 0, rows on bit 1), so lanes on the same node quad -
    // sorted particles put one to a few quads in a warp - hit four different
    // nodes in each atomic.  (Summing the lanes of a quad first with
    // match.any / redux.sync made this pass two to four times slower on B200.)
    if (act) {
      int c0, c1, r0, r1, vr[4], vz[4];
      deposit_nodes32(P, ir, iz, fr, fz, ur, uz, ig, lane & 3, c0, c1, r0, r1, vr, vz);
      const unsigned l0 = (unsigned)(r0 - w.row0), l1 = (unsigned)(r1 - w.row0);
      if (l0 < (unsigned)w.rows && l1 < (unsigned)w.rows) {
        const int k0 = (int)l0 * w.ws, k1 = (int)l1 * w.ws;
        int *n00 = w.rz + 2 * (k0 + c0), *n10 = w.rz + 2 * (k0 + c1);
        int *n01 = w.rz + 2 * (k1 + c0), *n11 = w.rz + 2 * (k1 + c1);
        atomicAdd(n00, vr[0]); atomicAdd(n00 + 1, vz[0]);
        atomicAdd(n10, vr[1]); atomicAdd(n10 + 1, vz[1]);
        atomicAdd(n01, vr[2]); atomicAdd(n01 + 1, vz[2]);
        atomicAdd(n11, vr[3]); atomicAdd(n11 + 1, vz[3]);
      } else {
        win_node(w, P, c0, r0, vr[0], vz[0]);
        win_node(w, P, c1, r0, vr[1], vz[1]);
        win_node(w, P, c0, r1, vr[2], vz[2]);
        win_node(w, P, c1, r1, vr[3], vz[3]);
      }
      wc_max = max(wc_max, max(c0, c1));   // (win_node may use the window for one row)
    }
  }
  // the window columns this warp touched, merged into the block's; the wall
  // losses of the warp
  wc_max = __reduce_max_sync(0xFFFFFFFFu, wc_max);
  if (lane == 0 && wc_max >= 0) atomicMax(box_cmax, wc_max);
  lost = __reduce_add_sync(0xFFFFFFFFu, lost);
  if (lane == 0 && lost) atomicAdd(&cnt->lost, (unsigned long long)lost);
}

// Add the window columns [0, bw) of every window row to the grid (one 64-bit
// atomic per nonzero node) and zero them for the next chunk.
__device__ __forceinline__ void flush32(const SimParams &P, const Win32 &w, int bw) {
  const int nb = bw > 0 ? bw * w.rows : 0;
  for (int i = threadIdx.x; i < nb; i += kBlock) {
    const int row = i / bw, col = i - row * bw;
    const int k = row * w.ws + col;
    const int2 v = reinterpret_cast<const int2 *>(w.rz)[k];
    const int vr = v.x, vz = v.y;
    if (vr | vz) {
      const int64_t g = (int64_t)(w.row0 + row) * P.ldj + col;
      if (vr) atomicAdd(P.Jr + g, (unsigned long long)(long long)vr);
      if (vz) atomicAdd(P.Jz + g, (unsigned long long)(long long)vz);
      reinterpret_cast<int2 *>(w.rz)[k] = make_int2(0, 0);
    }
  }
}

constexpr int kCandLanes = 8;     // collision candidates a warp of the pass takes at once

// FP32 particle pass of step `step` (modes as push32).  Its blocks first take
// the collision candidates queued by the previous pass, kCandLanes per warp,
// one per lane (a long serial chain each; a warp's chains share its issue but
// serialise their different collision branches, so a few per warp, not 32,
// keep the longest warp short), then all other particles in chunks of
// P.chunk handed out in order, so the blocks that ran candidates simply take
// fewer chunks.  Counters are committed by the field
// kernel of the next step.
template <int MODE>
__global__ void __launch_bounds__(kBlock, 4) k_pass32(SimParams P, State32 S, Fields<float> F,
                                                      SimCounters *cnt, int *queue,
                                                      const SimParams *__restrict__ Pg) {
  constexpr int mode = MODE;
  __shared__ __align__(16) int win_rz[2 * kWinNodes];
  __shared__ int win_row0, win_rows;
  __shared__ int box_cmax;                       // highest window column the chunk touched
  __shared__ long long chunk_at;
  const long long n0 = (long long)cnt->n_total;   // births of this pass land beyond
  const long long step = cnt->step;
  const int par = (int)(step & 1);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // the window starts zeroed; each chunk's flush leaves it zeroed again
  for (int i = threadIdx.x; i < kWinNodes; i += kBlock) reinterpret_cast<int2 *>(win_rz)[i] = make_int2(0, 0);
  const int ws = win_stride(P.nr);
  const int maxrows = min(kWinNodes / ws, P.nz);
  const int chunk = P.chunk;
  const long long nchunk = (n0 + chunk - 1) / chunk;
  // thread 0 claims the block's next chunk (index and window rows) a chunk
  // ahead and has its state brought into L2 meanwhile; the first one before
  // the candidates, so that it has their time to arrive
  long long next_ch = 0;
  int next_row0 = 0, next_rows = 0;
  if (threadIdx.x == 0) {
    next_ch = (long long)atomicAdd(&cnt->chunk_next, 1ull);
    if (next_ch < nchunk) prefetch_chunk32(S, next_ch * chunk, min((next_ch + 1) * chunk, n0));
  }
  if (mode != 1) {
    const long long nq = (long long)cnt->n_cand[par ^ 1];
    const int *qin = queue + (long long)(par ^ 1) * P.cap;
    // kCandLanes candidates per warp, one per lane
    unsigned lost = 0;
    if (lane < kCandLanes)
      for (long long k = ((long long)blockIdx.x * (kBlock / 32) + warp) * kCandLanes + lane; k < nq;
           k += (long long)gridDim.x * (kBlock / 32) * kCandLanes)
        candidate32(Pg, F, S, cnt, queue, qin[k], step, mode, true, n0, lost);
    if (lost) atomicAdd(&cnt->lost, (unsigned long long)lost);
  }
  if (threadIdx.x == 0 && next_ch < nchunk) chunk_rows32(P, S, n0, chunk, next_ch, maxrows, next_row0, next_rows);
  for (;;) {
    if (threadIdx.x == 0) {
      chunk_at = next_ch;
      win_row0 = next_row0;
      win_rows = next_rows;
      box_cmax = -1;
    }
    __syncthreads();
    const long long ch = chunk_at;
    if (ch >= nchunk) break;
    // thread 0 claims the next chunk now; the claim's result is first used
    // after this chunk, so its round trip overlaps the chunk's work instead
    // of holding the block at the barrier above
    if (threadIdx.x == 0) next_ch = (long long)atomicAdd(&cnt->chunk_next, 1ull);
    // 32-bit slot indices: the capacity is below 2^31
    const int beg = (int)(ch * chunk), end = (int)min((long long)beg + chunk, n0);
    const Win32 w{win_rz, win_row0, win_rows, ws};
    chunk32<MODE>(P, S, F, cnt, queue, step, beg, end, w, &box_cmax);
    if (threadIdx.x == 0 && next_ch < nchunk) {
      prefetch_chunk32(S, next_ch * chunk, min((next_ch + 1) * chunk, n0));
      chunk_rows32(P, S, n0, chunk, next_ch, maxrows, next_row0, next_rows);
    }
    __syncthreads();
    flush32(P, w, box_cmax + 1);
    __syncthreads();
  }
}

// ------------------------------------------------------- batched FP32 pass
// One cell of a batch as the batched FP32 pass sees it (global memory): its
// parameters with the current buffer 0 / 1 as the deposit target, its two
// state buffers, counters, candidate queues and fields.
struct BatchCell32 {
  SimParams P[2];
  State32 S[2];
  SimCounters *cnt;
  int *queue;
  Fields<float> F[2];         // field buffers 0 / 1 (the pass into current buffer jb reads F[jb])
};

// The FP32 pass of one step for every cell of a batch in one launch: each
// block reads the cells' counters and forms the prefix sums of their
// collision candidates and chunks; the candidates of all cells go first, one
// per warp, then the blocks take (cell, chunk) work items from one counter
// (*chunk_next, zeroed before the launch), copying the cell's parameters into
// shared memory when the cell changes.  Every cell gives what its own
// k_pass32 gives.
__global__ void __launch_bounds__(kBlock, 4) k_batch_pass32(const BatchCell32 *__restrict__ cells,
                                                            int ncell, int cur, int jb,
                                                            unsigned long long *chunk_next) {
  constexpr int mode = 0;        // a batch only takes whole steps
  __shared__ __align__(16) int win_rz[2 * kWinNodes];
  __shared__ int win_row0, win_rows, box_cmax, cell_at;
  __shared__ long long chunk_at;
  __shared__ long long cand_pre[kMaxBatch + 1], chunk_pre[kMaxBatch + 1];
  __shared__ __align__(16) unsigned char sP_raw[sizeof(SimParams)];
  SimParams &sP = *reinterpret_cast<SimParams *>(sP_raw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kWinNodes; i += kBlock) reinterpret_cast<int2 *>(win_rz)[i] = make_int2(0, 0);
  // per-cell candidates (of the previous pass) and chunks, then prefix sums
  for (int c = threadIdx.x; c < ncell; c += kBlock) {
    const SimCounters *cc = cells[c].cnt;
    const long long step = cc->step;
    cand_pre[c + 1] = mode != 1 ? (long long)cc->n_cand[(int)(step & 1) ^ 1] : 0;
    const long long n0 = (long long)cc->n_total;
    const int chunk = cells[c].P[jb].chunk;
    chunk_pre[c + 1] = (n0 + chunk - 1) / chunk;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    cand_pre[0] = 0; chunk_pre[0] = 0;
    for (int c = 0; c < ncell; ++c) {
      cand_pre[c + 1] += cand_pre[c];
      chunk_pre[c + 1] += chunk_pre[c];
    }
  }
  __syncthreads();
  const long long nq = cand_pre[ncell], nchunk = chunk_pre[ncell];
  // (cell, chunk) work items; the block's first one is claimed (and its state
  // brought into L2) before the candidates
  long long next = 0;
  int next_c = -1, next_row0 = 0, next_rows = 0;
  auto resolve = [&]() {         // thread 0: the cell and window rows of the claimed item
    if (next < nchunk) {
      next_c = cell_of_item(chunk_pre, ncell, next);
      const BatchCell32 &C = cells[next_c];
      const SimParams &Pc = C.P[jb];
      const int ws = win_stride(Pc.nr), maxrows = min(kWinNodes / ws, Pc.nz);
      const long long n0c = (long long)C.cnt->n_total, chc = next - chunk_pre[next_c];
      prefetch_chunk32(C.S[cur], chc * Pc.chunk, min((chc + 1) * Pc.chunk, n0c));
      chunk_rows32(Pc, C.S[cur], n0c, Pc.chunk, chc, maxrows, next_row0, next_rows);
    }
  };
  if (threadIdx.x == 0) {
    next = (long long)atomicAdd(chunk_next, 1ull);
    resolve();
    cell_at = -1;
  }
  // one candidate per lane (the chains of a warp share its instruction issue)
  for (long long k = ((long long)blockIdx.x * (kBlock / 32) + warp) * 32 + lane; k < nq;
       k += (long long)gridDim.x * kBlock) {
    const int c = cell_of_item(cand_pre, ncell, k);
    const BatchCell32 &C = cells[c];
    SimCounters *cc = C.cnt;
    const long long step = cc->step;
    const int *qin = C.queue + (long long)((int)(step & 1) ^ 1) * C.P[jb].cap;
    unsigned lost = 0;
    candidate32(&C.P[jb], C.F[jb], C.S[cur], cc, C.queue, qin[k - cand_pre[c]], step, mode, true,
                (long long)cc->n_total, lost);
    if (lost) atomicAdd(&cc->lost, (unsigned long long)lost);
  }
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      chunk_at = next;
      win_row0 = next_row0;
      win_rows = next_rows;
      box_cmax = -1;
    }
    __syncthreads();
    const long long g = chunk_at;
    if (g >= nchunk) break;
    const int c = cell_of_item(chunk_pre, ncell, g);
    if (c != cell_at) {          // this block's first chunk of cell c: its parameters
      const uint32_t *src = reinterpret_cast<const uint32_t *>(&cells[c].P[jb]);
      uint32_t *dst = reinterpret_cast<uint32_t *>(sP_raw);
      for (int i = threadIdx.x; i < (int)(sizeof(SimParams) / 4); i += kBlock) dst[i] = src[i];
      __syncthreads();
      if (threadIdx.x == 0) cell_at = c;
    }
    // the next item is claimed now and resolved after this one, so the
    // claim's round trip and the loads it leads to overlap the chunk's work
    if (threadIdx.x == 0 && next < nchunk) next = (long long)atomicAdd(chunk_next, 1ull);
    const BatchCell32 &C = cells[c];
    SimCounters *cc = C.cnt;
    const long long n0 = (long long)cc->n_total, step = cc->step;
    const int chunk = sP.chunk;
    const long long ch = g - chunk_pre[c];
    const int beg = (int)(ch * chunk), end = (int)min((long long)beg + chunk, n0);
    const Win32 w{win_rz, win_row0, win_rows, win_stride(sP.nr)};
    chunk32<0>(sP, C.S[cur], C.F[jb], cc, C.queue, step, beg, end, w, &box_cmax);
    if (threadIdx.x == 0) resolve();
    __syncthreads();
    flush32(sP, w, box_cmax + 1);
  }
}

// The collisions still queued by the last FP32 pass, without the next push
// (before an observation of the state): MCC at the end of that step and the
// secondaries' birth; the pending flags are cleared.
__global__ void __launch_bounds__(kMccBlock) k_collide32(const SimParams *__restrict__ Pg,
                                                         State32 S, Fields<float> F,
                                                         SimCounters *cnt, int *queue) {
  const SimParams &P = *Pg;
  const long long n0 = (long long)cnt->n_total;
  const long long step = cnt->step;
  const int par = (int)(step & 1);
  const long long nq = (long long)cnt->n_cand[par];
  const int *qu = queue + (long long)par * P.cap;
  unsigned lost = 0;              // (no push here: nothing reaches the wall)
  for (long long k = blockIdx.x * (long long)kMccBlock + threadIdx.x; k < nq;
       k += (long long)gridDim.x * kMccBlock)
    candidate32(Pg, F, S, cnt, queue, qu[k], step, 0, false, n0, lost);
}

// k_collide32 for every cell of a batch in one launch (before the batch's
// sort): the cells' queued collisions in one range by prefix sums, one per
// lane; each cell's are those its own k_collide32 would apply.
__global__ void __launch_bounds__(kMccBlock) k_batch_collide32(const BatchCell32 *__restrict__ cells,
                                                               int ncell, int cur) {
  __shared__ long long pre[kMaxBatch + 1];
  for (int c = threadIdx.x; c < ncell; c += blockDim.x) {
    const SimCounters *cc = cells[c].cnt;
    pre[c + 1] = (long long)cc->n_cand[(int)(cc->step & 1)];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    pre[0] = 0;
    for (int c = 0; c < ncell; ++c) pre[c + 1] += pre[c];
  }
  __syncthreads();
  const long long nq = pre[ncell];
  for (long long k = blockIdx.x * (long long)kMccBlock + threadIdx.x; k < nq;
       k += (long long)gridDim.x * kMccBlock) {
    const int c = cell_of_item(pre, ncell, k);
    const BatchCell32 &C = cells[c];
    SimCounters *cc = C.cnt;
    const long long step = cc->step;
    const int *qu = C.queue + (long long)(int)(step & 1) * C.P[0].cap;
    unsigned lost = 0;
    candidate32(&C.P[0], C.F[0], C.S[cur], cc, C.queue, qu[k - pre[c]], step, 0, false,
                (long long)cc->n_total, lost);
  }
}

// every cell's collision queue of parity q emptied, after its collisions ran
template <typename Cell>
__global__ void k_batch_clear_cand(const Cell *__restrict__ cells, int ncell, int q) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x)
    cells[c].cnt->n_cand[q] = 0;
}

// ------------------------------------------------------------- FDTD
// FP32 form (cnt given): commit the previous pass and open step s - the
// births of the last pass join the slots, the queue that pass consumed is
// emptied, the chunk counter rewinds; no other kernel runs meanwhile
__device__ __forceinline__ void commit_pass32(SimCounters *cnt) {
  const long long ns = cnt->step + 1;
  const unsigned long long nt = cnt->n_total + cnt->n_births;
  cnt->n_total = nt < cnt->cap ? nt : cnt->cap;
  cnt->n_births = 0;
  cnt->n_cand[ns & 1] = 0;
  cnt->chunk_next = 0;
  cnt->step = ns;
}

// The field sub-cycle of one step for fdtd_ratio 1: one warp per patch of R
// rows (fdtd_tma.cuh).
template <typename T, int R>
__global__ void __launch_bounds__(32 * kTmaWarps, 2) k_sim_fdtd_tma(const __grid_constant__ FdtdInst I,
                                                                SimCounters *cnt) {
  if (cnt && blockIdx.x == 0 && threadIdx.x == 0) commit_pass32(cnt);
  fdtd_warp_body<T, R>(FdtdWork{&I, nullptr, I.ntiles});
}

// The field update of every cell of a batch in one launch: the warps walk a
// table of (cell, tile) work items; FP32 form (commit given): the blocks first
// commit the previous pass of every cell.
template <typename T, int R>
__global__ void __launch_bounds__(32 * kTmaWarps, 2) k_batch_fdtd_tma(const FdtdInst *insts,
                                                                  const int2 *table, int nitems,
                                                                  SimCounters *const *commit,
                                                                  int ninst) {
  if (commit && threadIdx.x == 0)
    for (int i = blockIdx.x; i < ninst; i += gridDim.x) commit_pass32(commit[i]);
  fdtd_warp_body<T, R>(FdtdWork{insts, table, nitems});
}

using SimFdtdTmaFn = void (*)(const FdtdInst, SimCounters *);
using BatchFdtdTmaFn = void (*)(const FdtdInst *, const int2 *, int, SimCounters *const *, int);

// the patch heights (rows) the field update is built for
__host__ __device__ constexpr bool tma_rows_ok(int rows) { return rows == 12 || rows == 16 || rows == 20; }

// the instance of each kernel, and its dynamic shared memory, for `rows`
template <typename T>
SimFdtdTmaFn sim_fdtd_tma_fn(int rows) {
  return rows == 12 ? k_sim_fdtd_tma<T, 12> : rows == 20 ? k_sim_fdtd_tma<T, 20> : k_sim_fdtd_tma<T, 16>;
}
template <typename T>
BatchFdtdTmaFn batch_fdtd_tma_fn(int rows) {
  return rows == 12 ? k_batch_fdtd_tma<T, 12> : rows == 20 ? k_batch_fdtd_tma<T, 20> : k_batch_fdtd_tma<T, 16>;
}
template <typename T>
size_t tma_block_bytes(int rows) {
  return rows == 12 ? TmaStage<T, 12>::block_bytes
                    : rows == 20 ? TmaStage<T, 20>::block_bytes : TmaStage<T, 16>::block_bytes;
}

// The general sub-cycle (fdtd_ratio > 1): one 32 x 32 patch per block
// (fdtd_tiled), from the fields `in` to the fields `out`.
template <typename T>
__global__ void __launch_bounds__(32 * kFdtdRows, 3) k_sim_fdtd(Fields<T> in, Fields<T> out,
                                                  const unsigned long long *Jr,
                                                  const unsigned long long *Jz,
                                                  unsigned long long *Jr_next,
                                                  unsigned long long *Jz_next, int nr, int nz,
                                                  int ldf, int ldj, FdtdCoef c, const double *invV, double mu,
                                                  double dt, int R, unsigned flags,
                                                  SimCounters *cnt, ExtraCurrent ion,
                                                  FieldQuads quads) {
  if (cnt && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && threadIdx.y == 0)
    commit_pass32(cnt);
  fdtd_tiled<T>(in.Er, in.Ez, in.H, out.Er, out.Ez, out.H, Jr, Jz, Jr_next, Jz_next, nr, nz, ldf, ldj,
                c, invV, mu, dt, R, flags, ion, quads);
}

// ---------------------------------------------------------- load/read

// one particle in SI (r, z [m], u = gamma v [m/s]) into the FP32 state; mark:
// the pushed-parity flag (the opposite of the parity of the pass that will
// push it first)
__device__ __forceinline__ void store32(State32 S, long long p, double r, double z, double ur,
                                        double ut, double uz, uint64_t id, int nr, int nz,
                                        double dr, double dz, double c, int mark) {
  const double R = r / dr, Z = z / dz;
  int ir = (int)floor(R), iz = (int)floor(Z);
  float fr = (float)(R - ir), fz = (float)(Z - iz);
  if (fr >= 1.f) { fr = 0.f; ir++; }
  if (fz >= 1.f) { fz = 0.f; iz++; }
  if (iz >= nz) { iz = nz - 1; fz = 0.99999994f; }
  const bool alive = r >= 0 && ir < nr && iz >= 0;
  S.a[p] = pack32(ir, iz, fr, fz, (float)(ur / c), alive, false, mark);
  S.b[p] = make_float2((float)(ut / c), (float)(uz / c));
  S.id[p] = id;
}

__device__ __forceinline__ void store64(State64 S, long long p, double r, double z, double ur,
                                        double ut, double uz, uint64_t id) {
  S.rz[p] = make_double2(r, z);
  S.urt[p] = make_double2(ur, ut);
  S.uz[p] = uz;
  S.id[p] = id;
}

__global__ void k_load64(State64 S, const double *r, const double *z, const double *ur,
                         const double *ut, const double *uz, const uint64_t *id, long long n) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x)
    store64(S, p, r[p], z[p], ur[p], ut[p], uz[p], id[p]);
}

__global__ void k_load32(State32 S, const double *r, const double *z, const double *ur,
                         const double *ut, const double *uz, const uint64_t *id, long long n,
                         int nr, int nz, double dr, double dz, double c, int mark) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x)
    store32(S, p, r[p], z[p], ur[p], ut[p], uz[p], id[p], nr, nz, dr, dz, c, mark);
}

// ------------------------------------------------------------ births
// Photoionization births on the device: per photon a photoelectron (photon
// energy minus the N K-shell binding, 410 eV as EB_14.csv's 409.9; direction
// density ~ (d . x)^2 about the polarisation x) and an isotropic 360 eV Auger
// electron, both at a Rayleigh(sigma_r) radius (inside the wall), uniform
// azimuth and uniform z; the state keeps the local (r, theta, z) frame of that
// azimuth.  The reference draws its births on the host (INCIDENCE1.m:51-158,
// with a Sauter photoelectron and a 383 eV Auger line); these are the
// workload's laws.  Draws: Philox keyed on (seed, photon index) with the
// reserved step word kBirthStream, apart from every simulation draw.
constexpr long long kBirthStream = -2;
constexpr double kKShellEv = 410.0, kAugerEv = 360.0;

template <int FORM>
__global__ void k_birth_photo(State64 S64, State32 S32, long long n_photo, double u_pe,
                              double u_au, double sigma_r, double r_max, double Lp,
                              uint64_t seed, uint64_t id_base, int nr, int nz, double dr,
                              double dz, double c) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n_photo;
       k += (long long)gridDim.x * blockDim.x) {
    const U2 d0 = draw2(seed, (uint64_t)k, kBirthStream, 0), d1 = draw2(seed, (uint64_t)k, kBirthStream, 1);
    const U2 d2 = draw2(seed, (uint64_t)k, kBirthStream, 2), d3 = draw2(seed, (uint64_t)k, kBirthStream, 3);
    const double r = fmin(sigma_r * sqrt(-2.0 * log1p(-d0.a)), r_max);
    const double z = d0.b * Lp;
    double sp, cp;
    sincos(2 * GASATT_PI * d1.a, &sp, &cp);                // azimuth of the birth point
    // photoelectron: mu = cos(angle to x), p(mu) ~ mu^2 -> mu = cbrt(2U - 1)
    const double mu = cbrt(2 * d1.b - 1), s = sqrt(fmax(0.0, 1 - mu * mu));
    double sps, cps;
    sincos(2 * GASATT_PI * d2.a, &sps, &cps);
    const double px = mu, py = s * cps, pz = s * sps;
    // Auger: isotropic
    const double ct = 2 * d2.b - 1, st = sqrt(fmax(0.0, 1 - ct * ct));
    double spa, cpa;
    sincos(2 * GASATT_PI * d3.a, &spa, &cpa);
    const double ax = st * cpa, ay = st * spa, az = ct;
    const double pr = u_pe * (px * cp + py * sp), pt = u_pe * (-px * sp + py * cp), pzz = u_pe * pz;
    const double ar = u_au * (ax * cp + ay * sp), at = u_au * (-ax * sp + ay * cp), azz = u_au * az;
    const long long p = 2 * k;
    if (FORM == 0) {
      store64(S64, p, r, z, pr, pt, pzz, id_base + (uint64_t)p);
      store64(S64, p + 1, r, z, ar, at, azz, id_base + (uint64_t)p + 1);
    } else {
      store32(S32, p, r, z, pr, pt, pzz, id_base + (uint64_t)p, nr, nz, dr, dz, c, 0);
      store32(S32, p + 1, r, z, ar, at, azz, id_base + (uint64_t)p + 1, nr, nz, dr, dz, c, 0);
    }
  }
}

__global__ void k_read64(State64 S, double *r, double *z, double *ur, double *ut, double *uz,
                         uint64_t *id, long long n) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    const double2 a = S.rz[p], b = S.urt[p];
    r[p] = a.x; z[p] = a.y; ur[p] = b.x; ut[p] = b.y; uz[p] = S.uz[p];
    id[p] = S.id[p];
  }
}

__global__ void k_read32(State32 S, double *r, double *z, double *ur, double *ut, double *uz,
                         uint64_t *id, long long n, double dr, double dz, double c) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    const uint4 A = S.a[p];
    const float2 B = S.b[p];
    if (A.x == kDead) { r[p] = -1.0; z[p] = 0; }
    else {
      r[p] = ((double)(A.x & 0xFFFFu) + (double)__uint_as_float(A.y & ~kSign)) * dr;
      z[p] = ((double)(A.x >> 16) + (double)__uint_as_float(A.z & ~kSign)) * dz;
    }
    ur[p] = (double)__uint_as_float(A.w) * c; ut[p] = (double)B.x * c; uz[p] = (double)B.y * c;
    id[p] = S.id[p];
  }
}

// ---------------------------------------------------------------- sort
// Counting sort by cell (z-major), dropping dead slots.  Order inside a cell
// is arbitrary; nothing downstream depends on it (random streams are keyed
// on particle ids and the deposit is an exact integer sum).
// sort key: the deposit node quad (ar, az) = cell shifted by half a cell, so
// that lanes of a warp share their four deposit nodes right after a sort;
// (nr + 1) x (nz + 1) bins
__device__ __forceinline__ int cell_of64(const State64 &S, long long p, int nr, int nz,
                                         double dr, double dz) {
  const double2 rz = S.rz[p];
  if (rz.x < 0) return -1;
  int ar = (int)floor(rz.x / dr - 0.5) + 1, az = (int)floor(rz.y / dz - 0.5) + 1;
  ar = min(max(ar, 0), nr);
  az = min(max(az, 0), nz);
  return ar + az * (nr + 1);
}
__device__ __forceinline__ int cell_of32(const State32 &S, long long p, int nr) {
  const uint4 A = S.a[p];
  if (A.x == kDead) return -1;
  const int ar = (int)(A.x & 0xFFFFu) + (__uint_as_float(A.y & ~kSign) >= 0.5f ? 1 : 0);
  const int az = (int)(A.x >> 16) + (__uint_as_float(A.z & ~kSign) >= 0.5f ? 1 : 0);
  return ar + az * (nr + 1);
}

// Runs of equal keys among the lanes of a warp (the particles are nearly in
// key order, so a warp holds few runs): a lane heads a run when its key
// differs from the lane below's; dead lanes (key -1) end runs.  For each lane:
// its run's head lane h and, at the head, the run's length.
__device__ __forceinline__ void key_runs(int c, int lane, int &h, int &len) {
  const int below = __shfl_up_sync(0xFFFFFFFFu, c, 1);
  const bool head = c >= 0 && (lane == 0 || below != c);
  const unsigned heads = __ballot_sync(0xFFFFFFFFu, head);
  const unsigned ends = __ballot_sync(0xFFFFFFFFu, head || c < 0);
  const unsigned up = lane == 31 ? 0u : ends & (0xFFFFFFFFu << (lane + 1));
  len = (up ? __ffs(up) - 1 : 32) - lane;
  const unsigned le = heads & (lane == 31 ? 0xFFFFFFFFu : ((2u << lane) - 1));
  h = le ? 31 - __clz(le) : lane;
}

// Each warp takes segments of kSortSeg particles (kSortSeg / 32 per lane,
// consecutive groups of 32), loading all of a segment's keys before using
// them, so that several loads per thread are in flight.
constexpr int kSortSeg = 128;

template <int FORM>
__global__ void k_sort_hist(State64 S64, State32 S32, const SimCounters *cnt, int nr, int nz,
                            double dr, double dz, int *count) {
  constexpr int G = kSortSeg / 32;
  const long long n0 = slots_in_use(cnt);
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x / 32);
  for (long long seg = (long long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
       seg * kSortSeg < n0; seg += warps) {
    int c[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const long long p = seg * kSortSeg + g * 32 + lane;
      c[g] = -1;
      if (p < n0) c[g] = FORM == 0 ? cell_of64(S64, p, nr, nz, dr, dz) : cell_of32(S32, p, nr);
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
      int h, len;
      key_runs(c[g], lane, h, len);
      if (c[g] >= 0 && h == lane) atomicAdd(count + c[g], len);
    }
  }
}

template <int FORM>
__global__ void k_sort_scatter(State64 A64, State64 B64, State32 A32, State32 B32,
                               SimCounters *cnt, int nr, int nz, double dr, double dz,
                               const int *offset, int *cursor) {
  constexpr int G = kSortSeg / 32;
  const long long n0 = slots_in_use(cnt);
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x / 32);
  for (long long seg = (long long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
       seg * kSortSeg < n0; seg += warps) {
    int c[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const long long p = seg * kSortSeg + g * 32 + lane;
      c[g] = -1;
      if (p < n0) c[g] = FORM == 0 ? cell_of64(A64, p, nr, nz, dr, dz) : cell_of32(A32, p, nr);
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const long long p = seg * kSortSeg + g * 32 + lane;
      int h, len;
      key_runs(c[g], lane, h, len);
      // the head claims its run's slots in the bin and hands the first one out
      long long first = 0;
      if (c[g] >= 0 && h == lane) first = (long long)offset[c[g]] + atomicAdd(cursor + c[g], len);
      first = __shfl_sync(0xFFFFFFFFu, first, h);
      if (c[g] < 0) continue;
      const long long dst = first + (lane - h);
      if (FORM == 0) {
        B64.rz[dst] = A64.rz[p]; B64.urt[dst] = A64.urt[p]; B64.uz[dst] = A64.uz[p];
        B64.id[dst] = A64.id[p];
      } else {
        B32.a[dst] = A32.a[p]; B32.b[dst] = A32.b[p]; B32.id[dst] = A32.id[p];
      }
    }
  }
}

// ------------------------------------------------------------ scan
// Exclusive prefix sum of n ints in one pass (decoupled look-back): each
// block takes a tile of kScanTile counts by ticket, so a tile's predecessors
// are always running or done; it publishes its tile total (flag 1), looks
// back over the predecessors' published totals until it meets an inclusive
// prefix (flag 2), publishes its own inclusive prefix and writes its tile.
// The look-back reads 32 predecessors at a time, one per lane of a warp.
// A published word is (flag << 62) | value, written in one 64-bit store.
// The look-back wait on a tile that has published nothing yet is bounded;
// past the bound the scan sets *err and takes 0 for the tiles it waited on.
constexpr int kScanThreads = 256, kScanItems = 16, kScanTile = kScanThreads * kScanItems;
constexpr unsigned kScanWaitLimit = 1u << 24;

struct ScanState {
  unsigned long long *tile;   // ceil(n / kScanTile) published words, zeroed before each scan
  unsigned *ticket;           // tile ticket, zeroed before each scan
  unsigned *err;
};

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.volatile.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan(const int *in, int *out, int n, ScanState S) {
  __shared__ int warp_sum[kScanThreads / 32];
  __shared__ unsigned tile_s;
  __shared__ long long excl_s;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) tile_s = atomicAdd(S.ticket, 1u);
  __syncthreads();
  const unsigned t = tile_s;
  const long long base = (long long)t * kScanTile + (long long)threadIdx.x * kScanItems;
  int v[kScanItems];
  int sum = 0;
  if (base + kScanItems <= n) {            // whole: four 16-byte loads (base is a multiple of 16)
#pragma unroll
    for (int k = 0; k < kScanItems; k += 4) {
      const int4 q = *reinterpret_cast<const int4 *>(in + base + k);
      v[k] = q.x; v[k + 1] = q.y; v[k + 2] = q.z; v[k + 3] = q.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) v[k] = base + k < n ? in[base + k] : 0;
  }
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) sum += v[k];
  // block scan of the thread sums
  int incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_sum[warp] = incl;
  __syncthreads();
  int wbase = 0, total = 0;
#pragma unroll
  for (int w = 0; w < kScanThreads / 32; ++w) {
    wbase += w < warp ? warp_sum[w] : 0;
    total += warp_sum[w];
  }
  if (warp == 0) {
    // warp-parallel look-back: lane i reads the word of tile p - i; the
    // aggregates up to the nearest inclusive prefix are summed in one go
    constexpr unsigned long long kVal = (1ull << 62) - 1;
    long long excl = 0;
    if (t == 0) {
      if (lane == 0) atomicExch(S.tile, (2ull << 62) | (unsigned long long)total);
    } else {
      if (lane == 0) atomicExch(S.tile + t, (1ull << 62) | (unsigned long long)total);
      bool failed = false;
      for (long long p = (long long)t - 1; p >= 0; p -= 32) {
        const long long q = p - lane;
        // before tile 0: an inclusive prefix of 0
        unsigned long long w = q >= 0 ? ld_volatile_u64(S.tile + q) : (2ull << 62);
        unsigned it = 0;
        while (__any_sync(0xFFFFFFFFu, (w >> 62) == 0) && ++it < kScanWaitLimit)
          if ((w >> 62) == 0) w = ld_volatile_u64(S.tile + q);
        if (__any_sync(0xFFFFFFFFu, (w >> 62) == 0)) { failed = true; break; }
        const unsigned inc = __ballot_sync(0xFFFFFFFFu, (w >> 62) == 2);
        const int stop = inc ? __ffs(inc) - 1 : 31;
        long long v = lane <= stop ? (long long)(w & kVal) : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
        excl += v;
        if (inc) break;
      }
      if (lane == 0) {
        if (failed) atomicOr(S.err, 1u);
        atomicExch(S.tile + t, (2ull << 62) | (unsigned long long)(excl + total));
      }
    }
    if (lane == 0) excl_s = excl;
  }
  __syncthreads();
  int run = (int)excl_s + wbase + incl - sum;
  if (base + kScanItems <= n) {
#pragma unroll
    for (int k = 0; k < kScanItems; k += 4) {
      int4 o;
      o.x = run; run += v[k];
      o.y = run; run += v[k + 1];
      o.z = run; run += v[k + 2];
      o.w = run; run += v[k + 3];
      *reinterpret_cast<int4 *>(out + base + k) = o;
    }
  } else {
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      if (base + k < n) out[base + k] = run;
      run += v[k];
    }
  }
}

__global__ void k_sort_finish(SimCounters *cnt, const int *offset, int ncell) {
  cnt->n_total = (unsigned long long)offset[ncell];
  cnt->n_births = 0;
  cnt->sorted_total = cnt->n_total;
}

// ---------------------------------------------------------- diagnostics
template <int FORM>
__global__ void k_diag(State64 S64, State32 S32, SimCounters *cnt, double c, double me,
                       double qe) {
  const long long n0 = slots_in_use(cnt);
  unsigned long long kin = 0, alive = 0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n0;
       p += (long long)gridDim.x * blockDim.x) {
    double u2;
    if (FORM == 0) {
      if (S64.rz[p].x < 0) continue;
      const double2 a = S64.urt[p];
      const double w = S64.uz[p];
      u2 = (a.x * a.x + a.y * a.y + w * w) / (c * c);
    } else {
      const uint4 A = S32.a[p];
      if (A.x == kDead) continue;
      const float2 B = S32.b[p];
      const double a = __uint_as_float(A.w), b = B.x, d = B.y;
      u2 = a * a + b * b + d * d;
    }
    const double g = sqrt(1 + u2);
    const double Eev = me * c * c * (u2 / (g + 1)) / qe;
    kin += (unsigned long long)__double2ll_rn(Eev * 65536.0);
    alive++;
  }
  for (int o = 16; o; o >>= 1) {
    kin += __shfl_down_sync(0xFFFFFFFFu, kin, o);
    alive += __shfl_down_sync(0xFFFFFFFFu, alive, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&cnt->kin_fx, kin);
    atomicAdd(&cnt->alive, alive);
  }
}

// trapezoid-weighted field energy (electricmagneticfield6.m:153-154),
// per-block partial sums in a fixed order
template <typename T>
__global__ void k_field_energy(const T *Er, const T *Ez, const T *H, int nr, int nz, int ld,
                               double dr, double dz, double *partial) {
  __shared__ double sh[kBlock];
  const int64_t nE = (int64_t)nr * (nz + 1), nZ = (int64_t)(nr + 1) * nz, nH = (int64_t)nr * nz;
  double acc[3] = {0, 0, 0};
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < nE + nZ + nH;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int f, ncol, nrow;
    int64_t k;
    double r0;
    const T *A;
    if (idx < nE) { f = 0; k = idx; ncol = nr; nrow = nz + 1; r0 = dr / 2; A = Er; }
    else if (idx < nE + nZ) { f = 0; k = idx - nE; ncol = nr + 1; nrow = nz; r0 = 0; A = Ez; }
    else { f = 1; k = idx - nE - nZ; ncol = nr; nrow = nz; r0 = dr / 2; A = H; }
    const int i = (int)(k % ncol), j = (int)(k / ncol);
    const double wi = (i == 0 || i == ncol - 1) ? 0.5 : 1.0;
    const double wj = (j == 0 || j == nrow - 1) ? 0.5 : 1.0;
    const double v = (double)A[i + (int64_t)j * ld];
    acc[f] += wi * wj * v * v * (r0 + i * dr) * dr * dz;
  }
  for (int f = 0; f < 2; ++f) {
    sh[threadIdx.x] = acc[f];
    __syncthreads();
    for (int s = kBlock / 2; s; s >>= 1) {
      if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x * 2 + f] = sh[0];
    __syncthreads();
  }
}

}  // namespace

// ================================================================ sim object
struct gasatt_sim {
  gasatt_ctx *ctx = nullptr;
  gasatt_sim_config cfg{};
  SimTables tabs;
  SimParams P{};
  int form = 0;
  // state (double-buffered for the sort)
  State64 s64[2]{};
  State32 s32[2]{};
  int cur = 0;
  // fields, double-buffered: the step of parity q reads buffer q and writes
  // buffer 1 - q (the field update keeps patches of the old fields while
  // others are written), so the fields of the current time are in buffer
  // host_step & 1
  void *Er[2] = {nullptr, nullptr}, *Ez[2] = {nullptr, nullptr}, *H[2] = {nullptr, nullptr};
  // field update of fdtd_ratio 1: the cell's descriptor for the steps of
  // parity 0 / 1 (tensor maps of the fields and current read, write-back
  // targets, tiles), the patch rows, the grid and its shared memory
  FdtdInst fdtd_inst[2];
  int tma_rows = 0;
  unsigned tma_grid = 0;
  size_t tma_smem = 0;
  // Internal grid layout: column-major like the reference's arrays, with row
  // strides padded so that every row starts on a 16-byte boundary (the field
  // update stages its tiles with TMA).  Er(i, j) at i + j ldf (j <= n_z),
  // Ez(i, j) at i + j ldf (i <= n_r), H(i, j) at i + j ldf; currents
  // J(i, j) at i + j ldj.  The padding stays zero.
  int ldf = 0, ldj = 0;
  // current accumulators, double-buffered: the field update of step s reads
  // buffer s & 1 and clears the other one, which the pass of step s fills
  unsigned long long *Jr[2] = {nullptr, nullptr}, *Jz[2] = {nullptr, nullptr};
  double *d_tab = nullptr;
  double *invV = nullptr;         // per column: 2^-S / shell volume
  double *fdtd_colc = nullptr;    // per column: {invV, Ez coefficients} (fdtd_column_table)
  SimCounters *cnt = nullptr;
  SimCounters *h_cnt = nullptr;   // pinned
  int *cell_count = nullptr, *cell_offset = nullptr, *cell_cursor = nullptr;
  // the sort's scan: one published word per tile of counts, then the tile ticket
  unsigned long long *scan_tiles = nullptr;
  int scan_ntiles_max = 0;
  double *partial = nullptr;
  int partial_blocks = 0;
  std::vector<void *> allocs;
  bool primed = false;
  int64_t host_step = 0;          // particle passes completed
  int64_t since_sort = 0;
  cudaGraphExec_t g_step[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [state buffer][step parity]
  cudaGraph_t gr_step[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};     // the same, not instantiated
  cudaGraphExec_t g_sort[2] = {nullptr, nullptr};
  cudaGraph_t gr_sort[2] = {nullptr, nullptr};       // the same, not instantiated
  double scale = 1.0;
  unsigned pass_grid = 0, mcc_grid = 0;
  int *queue = nullptr;           // collision candidates, two queues of capacity slots
  SimParams *d_P = nullptr;       // device copies of P with the current of buffer 0 / 1
  double *d_gas = nullptr;        // per-cell gas density (gasatt_sim_set_gas_density)
  double *d_ion_sig = nullptr;    // per-cell newborn-ion spread (gasatt_sim_set_gas_temperature)
  // ions (cfg.ion_capacity > 0): the store lives in P.ion; the ion current,
  // deposited by each ion push and held until the next, in fixed point with
  // the factor ion_scale (2^48 per q_e FN c, in both forms)
  unsigned long long *Jir = nullptr, *Jiz = nullptr;
  double ion_scale = 1.0;
  IonState ion_tmp{};             // scratch store the ions are sorted into before a push
  FieldQuads quads{};             // FP32 form: gather quads, written with the fields
  bool mcc_pending = false;       // the last pass's collisions are not applied yet
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;   // graph capture fork/join
  bool timing = false;
  // field update start/end, particle pass start/end, collision kernel start/end
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

namespace {

template <typename T>
int sim_alloc(gasatt_sim *s, T **p, size_t n) {
  cudaError_t e = cudaMalloc((void **)p, (n ? n : 1) * sizeof(T));
  if (e != cudaSuccess) return cuda_fail(s->ctx, e, "cudaMalloc");
  s->allocs.push_back((void *)*p);
  return GASATT_OK;
}

#define SIM_TRY(x) do { int rc__ = (x); if (rc__) return rc__; } while (0)

// bytes of one current grid (n_z rows of ldj 64-bit counters)
size_t jbytes(const gasatt_sim *s) { return (size_t)s->ldj * s->cfg.n_z * 8; }

FdtdCoef fdtd_coef(const gasatt_sim *s) {
  const auto &c = s->cfg;
  const double dt = c.dt / c.fdtd_ratio, eps = c.eps0;
  FdtdCoef fc;
  fc.dr = c.dr; fc.dz = c.dz; fc.PHIp = c.PHIp; fc.inv_scale = 1.0 / s->scale;
  fc.dt_eps = (dt / 2) / eps;
  fc.dt_eps_dz = (dt / 2) / (eps * c.dz);
  fc.axis = 4 * (dt / 2) / (eps * c.dr);
  fc.chr = fc.chz = 0;
  return fc;
}

// field sub-cycle of step with parity q: reads current buffer q, clears 1 - q
// field buffer k as the kernels take it
template <typename T>
Fields<T> fields_of(const gasatt_sim *s, int k) {
  return Fields<T>{(T *)s->Er[k], (T *)s->Ez[k], (T *)s->H[k]};
}
// the field buffer that holds the fields of the current time
inline int fcur(const gasatt_sim *s) { return (int)(s->host_step & 1); }

// field update of a step of parity q: reads field buffer q and current
// buffer q, writes field buffer 1 - q and clears current buffer 1 - q
int launch_fdtd(gasatt_sim *s, cudaStream_t st, int q) {
  const auto &c = s->cfg;
  const int nr = c.n_r, nz = c.n_z, R = c.fdtd_ratio;
  const FdtdCoef fc = fdtd_coef(s);
  const double dt = c.dt / R;
  // the held ion current, in the electron current's fixed-point units
  const ExtraCurrent ion{s->Jir, s->Jiz, s->scale / s->ion_scale};
  if (R == 1) {
    const dim3 block(32 * kTmaWarps);
    if (s->form == 0)
      sim_fdtd_tma_fn<double>(s->tma_rows)<<<s->tma_grid, block, s->tma_smem, st>>>(s->fdtd_inst[q], nullptr);
    else
      sim_fdtd_tma_fn<float>(s->tma_rows)<<<s->tma_grid, block, s->tma_smem, st>>>(s->fdtd_inst[q], s->cnt);
    s->ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(s->ctx, e, "fdtd launch");
    return GASATT_OK;
  }
  const int tile = fdtd_tile(R);
  const dim3 grid((nr + 1 + tile - 1) / tile, (nz + 1 + tile - 1) / tile);
  const dim3 block(32, kFdtdRows);
  auto k64 = k_sim_fdtd<double>;
  auto k32 = k_sim_fdtd<float>;
  if (s->form == 0)
    k64<<<grid, block, 0, st>>>(
        fields_of<double>(s, q), fields_of<double>(s, 1 - q), s->Jr[q], s->Jz[q], s->Jr[1 - q],
        s->Jz[1 - q], nr, nz, s->ldf, s->ldj, fc, s->invV, c.mu0, dt, R, c.flags, nullptr, ion, FieldQuads{});
  else
    k32<<<grid, block, 0, st>>>(
        fields_of<float>(s, q), fields_of<float>(s, 1 - q), s->Jr[q], s->Jz[q], s->Jr[1 - q],
        s->Jz[1 - q], nr, nz, s->ldf, s->ldj, fc, s->invV, c.mu0, dt, R, c.flags, s->cnt, ion, s->quads);
  s->ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(s->ctx, e, "fdtd launch");
  return GASATT_OK;
}

// particle pass; its collision candidates (mode 0) go to queue q, its
// current to buffer jb; it gathers from field buffer fb
int launch_pass(gasatt_sim *s, cudaStream_t st, int mode, int jb, int q, int fb) {
  SimParams P = s->P;
  P.Jr = s->Jr[jb];
  P.Jz = s->Jz[jb];
  const int b = s->cur;
  if (s->form == 0)
    k_pass64<<<s->pass_grid, kBlock, 0, st>>>(P, s->s64[b], fields_of<double>(s, fb), s->cnt,
                                              s->queue, mode, q);
  else
  {
    auto kern = mode == 0 ? k_pass32<0> : mode == 1 ? k_pass32<1> : k_pass32<2>;
    kern<<<s->pass_grid, kBlock, 0, st>>>(P, s->s32[b], fields_of<float>(s, fb), s->cnt, s->queue,
                                          s->d_P + jb);
  }
  s->ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(s->ctx, e, "particle pass launch");
  return GASATT_OK;
}

// the commit of the last pass (its parity q)
int launch_commit(gasatt_sim *s, cudaStream_t st, int q) {
  k_commit<<<1, 1, 0, st>>>(s->cnt, q);
  s->ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(s->ctx, e, "commit launch");
  return GASATT_OK;
}

// the collisions queued (parity q) by the last pass that used that parity
int launch_mcc(gasatt_sim *s, cudaStream_t st, int q) {
  const int b = s->cur;
  if (s->form == 0)
    k_mcc64<<<s->mcc_grid, kMccBlock, 0, st>>>(s->P, s->s64[b], s->cnt, s->queue, q);
  else
    k_collide32<<<s->mcc_grid, kMccBlock, 0, st>>>(s->d_P, s->s32[b], fields_of<float>(s, fcur(s)),
                                                   s->cnt, s->queue);
  s->ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(s->ctx, e, "collision launch");
  return GASATT_OK;
}

// Apply the collisions still queued by the last pass, so that the particle
// state and the counters are complete (before a sort, a read, diagnostics or
// the end of a run).  The queue is emptied afterwards, so the collision kernel
// of the next step graph finds nothing to redo.
int flush_collisions(gasatt_sim *s) {
  if (!s->mcc_pending) return GASATT_OK;
  const int q = (int)((s->host_step - 1) & 1);
  cudaStream_t st = s->ctx->stream;
  if (s->form == 0) SIM_TRY(launch_commit(s, st, q));
  SIM_TRY(launch_mcc(s, st, q));
  GASATT_CUDA(s->ctx, cudaMemsetAsync(&s->cnt->n_cand[q], 0, sizeof(unsigned long long), st));
  s->mcc_pending = false;
  return GASATT_OK;
}

// exclusive prefix sum of n counts (k_scan), its tile words and ticket cleared first
int launch_scan(gasatt_sim *s, cudaStream_t st, const int *in, int *out, int n) {
  const int ntiles = (n + kScanTile - 1) / kScanTile;
  if (ntiles > s->scan_ntiles_max) return fail(s->ctx, GASATT_E_ARG, "scan longer than its tile words");
  GASATT_CUDA(s->ctx, cudaMemsetAsync(s->scan_tiles, 0, ((size_t)ntiles + 1) * 8, st));
  k_scan<<<ntiles, kScanThreads, 0, st>>>(
      in, out, n, ScanState{s->scan_tiles, reinterpret_cast<unsigned *>(s->scan_tiles + ntiles), &s->cnt->scan_err});
  s->ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(s->ctx, e, "scan launch");
  return GASATT_OK;
}

// Ion push after step host_step when it completes a sub-cycle.  Collisions
// still queued are applied first, so that the ions born in the step just
// taken are pushed with the others.
int launch_ion_push(gasatt_sim *s, cudaStream_t st) {
  SIM_TRY(flush_collisions(s));
  const auto &c = s->cfg;
  const int nbin = (c.n_r + 1) * (c.n_z + 1);
  const unsigned g = grid_for(c.ion_capacity, kBlock) < s->pass_grid ? grid_for(c.ion_capacity, kBlock) : s->pass_grid;
  // sort the store into the scratch store (the electrons' sort buffers are free here)
  GASATT_CUDA(s->ctx, cudaMemsetAsync(s->cell_count, 0, (size_t)(nbin + 1) * 4, st));
  GASATT_CUDA(s->ctx, cudaMemsetAsync(s->cell_cursor, 0, (size_t)nbin * 4, st));
  k_ion_hist<<<g, kBlock, 0, st>>>(s->P.ion, s->cnt, c.ion_capacity, c.n_r, c.n_z, c.dr, c.dz, s->cell_count);
  SIM_TRY(launch_scan(s, st, s->cell_count, s->cell_offset, nbin + 1));
  k_ion_scatter<<<g, kBlock, 0, st>>>(s->P.ion, s->ion_tmp, s->cnt, c.ion_capacity, c.n_r, c.n_z, c.dr,
                                      c.dz, s->cell_offset, s->cell_cursor);
  k_ion_sort_finish<<<1, 1, 0, st>>>(s->cnt, s->cell_offset, nbin);
  s->ctx->launches += 3;
  GASATT_CUDA(s->ctx, cudaMemsetAsync(s->Jir, 0, jbytes(s), st));
  GASATT_CUDA(s->ctx, cudaMemsetAsync(s->Jiz, 0, jbytes(s), st));
  SimParams PI = s->P;
  PI.dt = c.dt * c.ion_subcycle;
  PI.qm_dt2 = c.q_e / c.m_ion * PI.dt / 2;
  PI.dep = s->ion_scale;
  PI.Jr = s->Jir; PI.Jz = s->Jiz;
  if (s->form == 0)
    k_ion_push<double><<<g, kBlock, 0, st>>>(PI, fields_of<double>(s, fcur(s)), s->cnt, s->ion_tmp);
  else
    k_ion_push<float><<<g, kBlock, 0, st>>>(PI, fields_of<float>(s, fcur(s)), s->cnt, s->ion_tmp);
  s->ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(s->ctx, e, "ion push launch");
  return GASATT_OK;
}

bool ion_push_due(const gasatt_sim *s) {
  return s->cfg.ion_capacity > 0 && s->host_step % s->cfg.ion_subcycle == 0;
}

// sort from buffer `from` into 1 - from
int launch_sort(gasatt_sim *s, cudaStream_t st, int from) {
  const auto &c = s->cfg;
  const int ncell = (c.n_r + 1) * (c.n_z + 1);    // sort bins
  GASATT_CUDA(s->ctx, cudaMemsetAsync(s->cell_count, 0, (size_t)(ncell + 1) * 4, st));
  GASATT_CUDA(s->ctx, cudaMemsetAsync(s->cell_cursor, 0, (size_t)ncell * 4, st));
  const unsigned g = s->pass_grid;
  if (s->form == 0)
    k_sort_hist<0><<<g, kBlock, 0, st>>>(s->s64[from], s->s32[from], s->cnt, c.n_r, c.n_z, c.dr, c.dz, s->cell_count);
  else
    k_sort_hist<1><<<g, kBlock, 0, st>>>(s->s64[from], s->s32[from], s->cnt, c.n_r, c.n_z, c.dr, c.dz, s->cell_count);
  s->ctx->launches++;
  SIM_TRY(launch_scan(s, st, s->cell_count, s->cell_offset, ncell + 1));
  if (s->form == 0)
    k_sort_scatter<0><<<g, kBlock, 0, st>>>(s->s64[from], s->s64[1 - from], s->s32[from], s->s32[1 - from],
                                            s->cnt, c.n_r, c.n_z, c.dr, c.dz, s->cell_offset, s->cell_cursor);
  else
    k_sort_scatter<1><<<g, kBlock, 0, st>>>(s->s64[from], s->s64[1 - from], s->s32[from], s->s32[1 - from],
                                            s->cnt, c.n_r, c.n_z, c.dr, c.dz, s->cell_offset, s->cell_cursor);
  s->ctx->launches++;
  k_sort_finish<<<1, 1, 0, st>>>(s->cnt, s->cell_offset, ncell);
  s->ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(s->ctx, e, "sort launch");
  return GASATT_OK;
}

void drop_graphs(gasatt_sim *s) {
  for (int i = 0; i < 2; ++i) {
    for (int q = 0; q < 2; ++q) {
      if (s->g_step[i][q]) cudaGraphExecDestroy(s->g_step[i][q]);
      s->g_step[i][q] = nullptr;
      if (s->gr_step[i][q]) cudaGraphDestroy(s->gr_step[i][q]);
      s->gr_step[i][q] = nullptr;
    }
    if (s->g_sort[i]) cudaGraphExecDestroy(s->g_sort[i]);
    s->g_sort[i] = nullptr;
    if (s->gr_sort[i]) cudaGraphDestroy(s->gr_sort[i]);
    s->gr_sort[i] = nullptr;
  }
}

// host_step starts over at 0: the fields of the current time move to field
// buffer 0 (they are in buffer host_step & 1)
int restart_steps(gasatt_sim *s, cudaStream_t st) {
  if (fcur(s) != 0) {
    const size_t esz = s->form == 0 ? 8 : 4, nz = (size_t)s->cfg.n_z, ld = (size_t)s->ldf;
    GASATT_CUDA(s->ctx, cudaMemcpyAsync(s->Er[0], s->Er[1], ld * (nz + 1) * esz, cudaMemcpyDeviceToDevice, st));
    GASATT_CUDA(s->ctx, cudaMemcpyAsync(s->Ez[0], s->Ez[1], ld * nz * esz, cudaMemcpyDeviceToDevice, st));
    GASATT_CUDA(s->ctx, cudaMemcpyAsync(s->H[0], s->H[1], ld * nz * esz, cudaMemcpyDeviceToDevice, st));
  }
  s->host_step = 0;
  return GASATT_OK;
}

// A fresh population of n particles sits in state buffer 0: counters, current
// buffers and the step bookkeeping start over.
int sim_reset(gasatt_sim *s, int64_t n) {
  gasatt_ctx *ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  SimCounters zc{};
  zc.n_total = (unsigned long long)n;
  zc.step = -1;
  zc.cap = (unsigned long long)s->cfg.capacity;
  GASATT_CUDA(ctx, cudaMemcpyAsync(s->cnt, &zc, sizeof(zc), cudaMemcpyHostToDevice, st));
  for (int q = 0; q < 2; ++q) {
    GASATT_CUDA(ctx, cudaMemsetAsync(s->Jr[q], 0, jbytes(s), st));
    GASATT_CUDA(ctx, cudaMemsetAsync(s->Jz[q], 0, jbytes(s), st));
  }
  if (s->Jir) {                    // a new run: no ions, no ion current
    GASATT_CUDA(ctx, cudaMemsetAsync(s->Jir, 0, jbytes(s), st));
    GASATT_CUDA(ctx, cudaMemsetAsync(s->Jiz, 0, jbytes(s), st));
  }
  SIM_TRY(restart_steps(s, st));
  GASATT_CUDA(ctx, cudaStreamSynchronize(st));
  s->primed = false;
  s->mcc_pending = false;
  s->since_sort = 0;
  return GASATT_OK;
}

// Null-collision bound for a peak gas density n_max: nu_max = n_max *
// max(sigma_tot v), P_null = 1 - exp(-nu_max dt), and the integer threshold
// of the candidate test on the 52-bit draw.
void set_collision_bound(gasatt_sim *s, double n_max) {
  SimParams &P = s->P;
  P.nu_max = n_max * s->tabs.sigv_max;
  P.P_null = -std::expm1(-P.nu_max * s->cfg.dt);
  // largest count of 52-bit draws b with (2b+1) 2^-53 < P_null (exact in double)
  uint64_t t = (uint64_t)std::floor(P.P_null * 0x1.0p52);
  while ((2.0 * (double)t + 1.0) * 0x1.0p-53 < P.P_null) ++t;
  while (t > 0 && !((2.0 * (double)(t - 1) + 1.0) * 0x1.0p-53 < P.P_null)) --t;
  P.cand_below = t;
}

// cuTensorMapEncodeTiled from the driver (looked up once)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// A 2D tensor map over a w x h grid of elements with row stride ld_bytes
// (a multiple of 16), box bw x bh; out-of-bounds boxes fill with zeros.
int encode_map(gasatt_sim *s, CUtensorMap *m, CUtensorMapDataType type, void *base, int w, int h,
               size_t ld_bytes, int bw, int bh) {
  auto enc = tensor_map_encoder();
  if (!enc) return fail(s->ctx, GASATT_E_CUDA, "cuTensorMapEncodeTiled not available from the driver");
  const cuuint64_t dims[2] = {(cuuint64_t)w, (cuuint64_t)h};
  const cuuint64_t strides[1] = {(cuuint64_t)ld_bytes};
  const cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
  const cuuint32_t es[2] = {1, 1};
  const CUresult r = enc(m, type, 2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return fail(s->ctx, GASATT_E_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return GASATT_OK;
}

// The field update of fdtd_ratio 1: patch rows, tiles, grid, shared memory
// and the tensor maps of the fields and of both current buffers.
template <typename T>
int setup_fdtd_tma(gasatt_sim *s, int nsm) {
  const auto &c = s->cfg;
  const int ph = c.fdtd_tile_rows > 0 ? c.fdtd_tile_rows : 12;
  if (!tma_rows_ok(ph)) return fail(s->ctx, GASATT_E_ARG, "fdtd_tile_rows: 12, 16 or 20");
  s->tma_rows = ph;
  s->tma_smem = tma_block_bytes<T>(ph);
  const int tiles_x = (c.n_r + 1 + kTmaTileW - 1) / kTmaTileW;
  const int tiles_y = (c.n_z + 1 + (ph - 2 * kTmaHalo) - 1) / (ph - 2 * kTmaHalo);
  const int ntiles = tiles_x * tiles_y;
  const SimFdtdTmaFn kern = sim_fdtd_tma_fn<T>(ph);
  GASATT_CUDA(s->ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)s->tma_smem));
  int occ = 0;
  GASATT_CUDA(s->ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 32 * kTmaWarps,
                                                                    s->tma_smem));
  if (occ < 1) return fail(s->ctx, GASATT_E_ARG, "field update: patch does not fit in shared memory");
  const long long slots = (long long)nsm * occ, blocks = (ntiles + kTmaWarps - 1) / kTmaWarps;
  s->tma_grid = (unsigned)(slots < blocks ? slots : blocks);
  const CUtensorMapDataType ft = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  const size_t ldb = (size_t)s->ldf * sizeof(T), ldjb = (size_t)s->ldj * 8;
  const int bw = TmaBox<T>::w;
  for (int q = 0; q < 2; ++q) {
    FdtdInst &I = s->fdtd_inst[q];
    std::memset(&I, 0, sizeof(I));
    TmaMaps &M = I.maps;
    SIM_TRY(encode_map(s, &M.er, ft, s->Er[q], c.n_r, c.n_z + 1, ldb, bw, ph));
    SIM_TRY(encode_map(s, &M.ez, ft, s->Ez[q], c.n_r + 1, c.n_z, ldb, bw, ph));
    SIM_TRY(encode_map(s, &M.h, ft, s->H[q], c.n_r, c.n_z, ldb, bw, ph));
    SIM_TRY(encode_map(s, &M.jr, CU_TENSOR_MAP_DATA_TYPE_INT64, s->Jr[q], c.n_r, c.n_z, ldjb, 34, ph));
    SIM_TRY(encode_map(s, &M.jz, CU_TENSOR_MAP_DATA_TYPE_INT64, s->Jz[q], c.n_r, c.n_z, ldjb, 34, ph));
    I.Er = s->Er[1 - q]; I.Ez = s->Ez[1 - q]; I.H = s->H[1 - q];
    I.Jr_next = s->Jr[1 - q]; I.Jz_next = s->Jz[1 - q];
    I.colc = s->fdtd_colc;
    I.xj = ExtraCurrent{s->Jir, s->Jiz, s->scale / s->ion_scale};
    I.q = sizeof(T) == 4 ? s->quads : FieldQuads{};
    I.c = fdtd_coef(s);
    const double h4 = c.dt / 4, h2 = c.dt / 2;
    I.chr4 = h4 / (c.mu0 * I.c.dr);
    I.chz4 = h4 / (c.mu0 * I.c.dz);
    I.chr2 = h2 / (c.mu0 * I.c.dr);
    I.chz2 = h2 / (c.mu0 * I.c.dz);
    I.nr = c.n_r; I.nz = c.n_z; I.ldf = s->ldf; I.ldj = s->ldj;
    I.flags = c.flags;
    I.tiles_x = tiles_x;
    I.ntiles = ntiles;
    I.err = &s->cnt->fdtd_err;
  }
  return GASATT_OK;
}

// device copies of P (current buffers 0 and 1) for the kernels that read it
// from global memory
int upload_params(gasatt_sim *s) {
  SimParams Pq[2] = {s->P, s->P};
  Pq[0].Jr = s->Jr[0]; Pq[0].Jz = s->Jz[0];
  Pq[1].Jr = s->Jr[1]; Pq[1].Jz = s->Jz[1];
  GASATT_CUDA(s->ctx, cudaMemcpy(s->d_P, Pq, sizeof(Pq), cudaMemcpyHostToDevice));
  return GASATT_OK;
}

// Start of a run: the particles at x^0 move to x^{1/2} and deposit j^{1/2}
// (no collision candidates; queue parity 1 is the one step 0 reads).
int sim_prime(gasatt_sim *s) {
  if (s->primed) return GASATT_OK;
  cudaStream_t st = s->ctx->stream;
  if (s->cfg.sort_period > 0) SIM_TRY(gasatt_sim_sort(s));
  SIM_TRY(launch_pass(s, st, 1, 0, 1, fcur(s)));   // (a half drift reads no field)
  if (s->form == 0) SIM_TRY(launch_commit(s, st, 1));
  s->primed = true;
  return GASATT_OK;
}

// Capture one step for state buffer b and step parity q:
//
//    [field update of step s]  ||  [collisions queued by pass s-1 (parity 1-q)]
//                      \\               /
//                   [particle pass s: kick, drift, deposit, queue q]
//
// The field update needs only the current of pass s-1 and the collisions only
// the particles, so the two run side by side.  Also one sort b -> 1-b.
int build_graphs(gasatt_sim *s) {
  // the field update goes on a higher-priority stream than the collision
  // branch, so its blocks are placed first when both are ready
  int lo_prio = 0, hi_prio = 0;
  cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
  cudaStream_t cs, side;
  GASATT_CUDA(s->ctx, cudaStreamCreateWithPriority(&cs, cudaStreamNonBlocking, hi_prio));
  GASATT_CUDA(s->ctx, cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, lo_prio));
  const int save = s->cur;
  const int64_t save_launch = s->ctx->launches;
  int rc = GASATT_OK;
  for (int b = 0; b < 2 && !rc; ++b) {
    cudaGraph_t g;
    s->cur = b;
    for (int q = 0; q < 2 && !rc; ++q) {
      GASATT_CUDA(s->ctx, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
      if (s->form == 1) {
        // FP32: the field kernel commits the previous pass, the pass runs the
        // previous step's collisions itself.  Timing: one event before, one
        // between and one after the two kernels (the pass's collisions have
        // no kernel of their own)
        cudaError_t e = cudaSuccess;
        if (s->timing) e = cudaEventRecordWithFlags(s->ev[0], cs, cudaEventRecordExternal);
        if (e == cudaSuccess) rc = launch_fdtd(s, cs, q);
        if (e == cudaSuccess && !rc && s->timing)
          e = cudaEventRecordWithFlags(s->ev[1], cs, cudaEventRecordExternal);
        if (e == cudaSuccess && !rc) rc = launch_pass(s, cs, 0, 1 - q, q, 1 - q);
        if (e == cudaSuccess && !rc && s->timing)
          e = cudaEventRecordWithFlags(s->ev[3], cs, cudaEventRecordExternal);
        cudaError_t e2 = cudaStreamEndCapture(cs, &g);
        if (!rc && e != cudaSuccess) rc = cuda_fail(s->ctx, e, "capture step");
        if (!rc && e2 != cudaSuccess) rc = cuda_fail(s->ctx, e2, "capture step");
        if (!rc) {
          e = cudaGraphInstantiate(&s->g_step[b][q], g, 0);
          if (e != cudaSuccess) rc = cuda_fail(s->ctx, e, "instantiate step");
        }
        if (e2 == cudaSuccess) {
          if (!rc) s->gr_step[b][q] = g; else cudaGraphDestroy(g);
        }
        continue;
      }
      cudaError_t e = cudaEventRecord(s->fork_ev, cs);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(side, s->fork_ev, 0);
      if (e == cudaSuccess && s->timing) e = cudaEventRecordWithFlags(s->ev[4], side, cudaEventRecordExternal);
      if (e == cudaSuccess) rc = launch_commit(s, side, 1 - q);
      if (e == cudaSuccess && !rc) rc = launch_mcc(s, side, 1 - q);
      if (e == cudaSuccess && !rc && s->timing) e = cudaEventRecordWithFlags(s->ev[5], side, cudaEventRecordExternal);
      if (e == cudaSuccess && !rc) e = cudaEventRecord(s->join_ev, side);
      if (e == cudaSuccess && !rc && s->timing) e = cudaEventRecordWithFlags(s->ev[0], cs, cudaEventRecordExternal);
      if (e == cudaSuccess && !rc) rc = launch_fdtd(s, cs, q);
      if (e == cudaSuccess && !rc && s->timing) e = cudaEventRecordWithFlags(s->ev[1], cs, cudaEventRecordExternal);
      if (e == cudaSuccess && !rc) e = cudaStreamWaitEvent(cs, s->join_ev, 0);
      if (e == cudaSuccess && !rc && s->timing) e = cudaEventRecordWithFlags(s->ev[2], cs, cudaEventRecordExternal);
      if (e == cudaSuccess && !rc) rc = launch_pass(s, cs, 0, 1 - q, q, 1 - q);
      if (e == cudaSuccess && !rc && s->timing) e = cudaEventRecordWithFlags(s->ev[3], cs, cudaEventRecordExternal);
      cudaError_t e2 = cudaStreamEndCapture(cs, &g);
      if (!rc && e != cudaSuccess) rc = cuda_fail(s->ctx, e, "capture step");
      if (!rc && e2 != cudaSuccess) rc = cuda_fail(s->ctx, e2, "capture step");
      if (!rc) {
        e = cudaGraphInstantiate(&s->g_step[b][q], g, 0);
        if (e != cudaSuccess) rc = cuda_fail(s->ctx, e, "instantiate step");
      }
      if (e2 == cudaSuccess) {
        if (!rc) s->gr_step[b][q] = g; else cudaGraphDestroy(g);
      }
    }
    if (rc) break;
    GASATT_CUDA(s->ctx, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    rc = launch_sort(s, cs, b);
    cudaError_t e = cudaStreamEndCapture(cs, &g);
    const bool captured = e == cudaSuccess;
    if (!rc && !captured) rc = cuda_fail(s->ctx, e, "capture sort");
    if (!rc) {
      e = cudaGraphInstantiate(&s->g_sort[b], g, 0);
      if (e != cudaSuccess) rc = cuda_fail(s->ctx, e, "instantiate sort");
    }
    if (captured) {
      if (!rc) s->gr_sort[b] = g; else cudaGraphDestroy(g);
    }
  }
  s->cur = save;
  s->ctx->launches = save_launch;
  cudaStreamDestroy(side);
  cudaStreamDestroy(cs);
  return rc;
}

}  // namespace

extern "C" {

int gasatt_sim_default_config(gasatt_sim_config *c) {
  if (!c) return GASATT_E_ARG;
  std::memset(c, 0, sizeof(*c));
  c->n_r = 256; c->n_z = 1024; c->dr = 5e-6; c->dz = 5e-6; c->dt = 1e-14;
  c->fdtd_ratio = 1;
  c->PHIp = 2 * GASATT_PI;
  c->FN = 1.0;
  c->gas_temperature = 300.0;
  c->kb = 1.380649e-23;
  c->gas_density = 133.322368 / (c->kb * 300.0);     // 1 Torr
  c->q_e = 1.602176634e-19; c->m_e = 9.1093837015e-31; c->c = 299792458.0;
  c->eps0 = 8.8541878128e-12; c->mu0 = 1.25663706212e-6;
  c->m_ion = 28.0134 * 1.66053906660e-27;
  c->precision = GASATT_FP32_SPLIT;
  c->capacity = 1 << 20;
  c->ion_capacity = 0;
  c->ion_subcycle = 50;
  c->seed = 0;
  c->flags = 0;
  c->sort_period = 20;
  c->secondaries = 1;
  c->table_n = 2048; c->table_emin_ev = 0.1; c->table_emax_ev = 30000.0;
  return GASATT_OK;
}

int gasatt_sim_create(gasatt_ctx *ctx, const gasatt_sim_config *cfg, const gasatt_tables *tab,
                      gasatt_sim **out) {
  if (!ctx || !cfg || !out) return GASATT_E_ARG;
  *out = nullptr;
  const gasatt_sim_config &c = *cfg;
  if (c.n_r < 2 || c.n_z < 2 || c.n_r > 65535 || c.n_z > 65535 ||
      (int64_t)(c.n_r + 1) * (c.n_z + 1) > 0x7FFFFFFFLL || !(c.dr > 0) || !(c.dz > 0) ||
      !(c.dt > 0) || c.fdtd_ratio < 1 || c.capacity < 1 || c.capacity > 0x7FFFFFFFLL ||
      (c.precision != GASATT_FP64 && c.precision != GASATT_FP32_SPLIT))
    return fail(ctx, GASATT_E_ARG, "sim config out of range");
  if (c.flags & ~(unsigned)(GASATT_Q_ER_END_COPY | GASATT_Q_EZ_AXIS_JSIGN | GASATT_Q_EZ_RSHIFT))
    return fail(ctx, GASATT_E_ARG, "the resident simulation accepts only the field quirk flags");
  if (c.pass_chunk < 0 || c.pass_chunk > kChunkMax || c.pass_chunk % kBlock)
    return fail(ctx, GASATT_E_ARG, "pass_chunk: a multiple of 256 in [256, 1792] (0: 1792)");
  if (c.fdtd_tile_rows < 0) return fail(ctx, GASATT_E_ARG, "fdtd_tile_rows: >= 0");
  if (c.gather < 0 || c.gather > 2) return fail(ctx, GASATT_E_ARG, "gather: 0 (auto), 1 (quads) or 2 (fields)");
  if (c.ion_capacity < 0 || (c.ion_capacity > 0 && (c.ion_subcycle < 1 || !(c.m_ion > 0) ||
                                                     !(c.gas_temperature >= 0))))
    return fail(ctx, GASATT_E_ARG, "ion species: ion_capacity >= 0, ion_subcycle >= 1, m_ion > 0");
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  gasatt_sim *s = new gasatt_sim();
  s->ctx = ctx;
  s->cfg = c;
  s->form = c.precision;
  std::string err;
  int rc = build_sim_tables(tab, c.table_n, c.table_emin_ev, c.table_emax_ev, c.gas_density, c.c,
                            c.m_e, c.q_e, s->tabs, err);
  if (rc) { delete s; return fail(ctx, rc, err); }
  const int64_t cap = c.capacity;
  const int nr = c.n_r, nz = c.n_z, nbin = (nr + 1) * (nz + 1);
  s->ldf = (nr + 1 + 3) & ~3;       // 16-byte rows for float and double
  s->ldj = (nr + 1) & ~1;           // 16-byte rows of 64-bit counters
  const size_t ncur = (size_t)s->ldj * nz;
  auto cleanup = [&](int code) { gasatt_sim_destroy(s); return code; };
  for (int b = 0; b < 2; ++b) {
    if (s->form == 0) {
      State64 &S = s->s64[b];
      if ((rc = sim_alloc(s, &S.rz, cap)) || (rc = sim_alloc(s, &S.urt, cap)) ||
          (rc = sim_alloc(s, &S.uz, cap)) || (rc = sim_alloc(s, &S.id, cap)))
        return cleanup(rc);
    } else {
      State32 &S = s->s32[b];
      if ((rc = sim_alloc(s, &S.a, cap)) || (rc = sim_alloc(s, &S.b, cap)) || (rc = sim_alloc(s, &S.id, cap)))
        return cleanup(rc);
    }
  }
  if ((rc = sim_alloc(s, &s->queue, 2 * (size_t)cap))) return cleanup(rc);
  if (c.ion_capacity > 0) {
    IonState &I = s->P.ion;
    const size_t ic = (size_t)c.ion_capacity;
    if ((rc = sim_alloc(s, &I.rz, ic)) || (rc = sim_alloc(s, &I.urt, ic)) ||
        (rc = sim_alloc(s, &I.uz, ic)) || (rc = sim_alloc(s, &I.id, ic)) ||
        (rc = sim_alloc(s, &I.q, ic)) || (rc = sim_alloc(s, &s->ion_tmp.rz, ic)) ||
        (rc = sim_alloc(s, &s->ion_tmp.urt, ic)) || (rc = sim_alloc(s, &s->ion_tmp.uz, ic)) ||
        (rc = sim_alloc(s, &s->ion_tmp.id, ic)) || (rc = sim_alloc(s, &s->ion_tmp.q, ic)) ||
        (rc = sim_alloc(s, &s->Jir, ncur)) || (rc = sim_alloc(s, &s->Jiz, ncur)))
      return cleanup(rc);
  }
  const size_t esz = s->form == 0 ? 8 : 4;
  double *tmpd;
  const size_t nfE = (size_t)s->ldf * (nz + 1), nfZ = (size_t)s->ldf * nz, nfH = (size_t)s->ldf * nz;
  if ((rc = sim_alloc(s, (char **)&s->Er[0], nfE * esz)) ||
      (rc = sim_alloc(s, (char **)&s->Ez[0], nfZ * esz)) ||
      (rc = sim_alloc(s, (char **)&s->H[0], nfH * esz)) ||
      (rc = sim_alloc(s, (char **)&s->Er[1], nfE * esz)) ||
      (rc = sim_alloc(s, (char **)&s->Ez[1], nfZ * esz)) ||
      (rc = sim_alloc(s, (char **)&s->H[1], nfH * esz)) ||
      (rc = sim_alloc(s, &s->Jr[0], ncur)) || (rc = sim_alloc(s, &s->Jz[0], ncur)) ||
      (rc = sim_alloc(s, &s->Jr[1], ncur)) || (rc = sim_alloc(s, &s->Jz[1], ncur)) ||
      (rc = sim_alloc(s, &s->cnt, 1)) || (rc = sim_alloc(s, &s->cell_count, (size_t)nbin + 1)) ||
      (rc = sim_alloc(s, &s->cell_offset, (size_t)nbin + 1)) ||
      (rc = sim_alloc(s, &s->cell_cursor, (size_t)nbin)) ||
      (rc = sim_alloc(s, &tmpd, (size_t)4 * c.table_n + (size_t)181 * c.table_n)))
    return cleanup(rc);
  s->d_tab = tmpd;
  if ((rc = sim_alloc(s, &s->invV, (size_t)nr)) || (rc = sim_alloc(s, &s->fdtd_colc, (size_t)3 * nr)))
    return cleanup(rc);
  // FP32 gather quads: 48 bytes more per cell written by every field update,
  // against nine fewer loads per electron; worth it where electrons are dense
  const bool quads = s->form == 1 &&
                     (c.gather == 1 || (c.gather == 0 && c.capacity >= 4 * (int64_t)(nr + 1) * (nz + 1)));
  if (quads) {
    if ((rc = sim_alloc(s, &s->quads.er, (size_t)(nr + 1) * nz)) ||
        (rc = sim_alloc(s, &s->quads.ez, (size_t)nr * (nz + 1))) ||
        (rc = sim_alloc(s, &s->quads.h, (size_t)(nr + 1) * (nz + 1))))
      return cleanup(rc);
    cudaMemset(s->quads.er, 0, (size_t)(nr + 1) * nz * 16);
    cudaMemset(s->quads.ez, 0, (size_t)nr * (nz + 1) * 16);
    cudaMemset(s->quads.h, 0, (size_t)(nr + 1) * (nz + 1) * 16);
  }
  s->scan_ntiles_max = (nbin + 1 + kScanTile - 1) / kScanTile;
  if ((rc = sim_alloc(s, &s->scan_tiles, (size_t)s->scan_ntiles_max + 1))) return cleanup(rc);
  s->partial_blocks = 296;
  if ((rc = sim_alloc(s, &s->partial, (size_t)2 * s->partial_blocks))) return cleanup(rc);
  if (cudaMallocHost((void **)&s->h_cnt, sizeof(SimCounters)) != cudaSuccess)
    return cleanup(fail(ctx, GASATT_E_CUDA, "cudaMallocHost"));
  // tables
  std::vector<double> host((size_t)4 * c.table_n + (size_t)181 * c.table_n);
  std::memcpy(host.data(), s->tabs.sig_el.data(), c.table_n * 8);
  std::memcpy(host.data() + c.table_n, s->tabs.sig_ion.data(), c.table_n * 8);
  std::memcpy(host.data() + 2 * c.table_n, s->tabs.sig_exc.data(), c.table_n * 8);
  std::memcpy(host.data() + 3 * c.table_n, s->tabs.edep.data(), c.table_n * 8);
  std::memcpy(host.data() + 4 * c.table_n, s->tabs.cdf.data(), (size_t)181 * c.table_n * 8);
  if (cudaMemcpy(s->d_tab, host.data(), host.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess)
    return cleanup(fail(ctx, GASATT_E_CUDA, "table upload"));
  // parameters
  SimParams &P = s->P;
  P.nr = nr; P.nz = nz; P.ldf = s->ldf; P.ldj = s->ldj; P.dr = c.dr; P.dz = c.dz; P.dt = c.dt; P.c = c.c; P.qe = c.q_e;
  P.me = c.m_e; P.mu0 = c.mu0; P.FN = c.FN; P.PHIp = c.PHIp; P.n_gas = c.gas_density;
  P.gas = nullptr;
  P.ion_sig = nullptr;
  P.Rp = nr * c.dr; P.Lp = nz * c.dz; P.kb = c.kb; P.m_ion = c.m_ion; P.T_gas = c.gas_temperature;
  P.chunk = c.pass_chunk > 0 ? c.pass_chunk : kChunkMax;
  P.seed = c.seed; P.pk = philox_keys(c.seed); P.secondaries = c.secondaries; P.cap = cap;
  P.ion_cap = c.ion_capacity;
  P.ion_sigma = c.ion_capacity > 0 ? std::sqrt(c.kb * c.gas_temperature / c.m_ion) : 0.0;
  P.qm_dt2 = -c.q_e / c.m_e * c.dt / 2;
  P.aE = (float)(-c.q_e * c.dt / (2 * c.m_e * c.c));
  P.aB = (float)(-c.q_e * c.dt * c.mu0 / (2 * c.m_e));
  P.hdr = (float)(c.c * c.dt / (2 * c.dr));
  P.hdz = (float)(c.c * c.dt / (2 * c.dz));
  // fixed point: FP64 |q FN v w| * scale <= 2^48; FP32 <= 2^20 (the int32
  // deposit window of a chunk of particles cannot overflow)
  const double qfc = c.q_e * std::fabs(c.FN) * c.c;
  s->scale = s->form == 0 ? std::ldexp(1.0, 48) / qfc : std::ldexp(1.0, 20) / qfc;
  P.dep = s->scale;
  P.depf = (float)(-c.q_e * c.FN * c.c * s->scale);
  s->ion_scale = std::ldexp(1.0, 48) / qfc;
  set_collision_bound(s, c.gas_density);
  P.sig = s->d_tab;
  P.edep = s->d_tab + 3 * c.table_n;
  P.cdf = s->d_tab + 4 * c.table_n;
  P.exc_kmin = s->tabs.exc_kmin;
  P.G = c.table_n; P.lnEmin = s->tabs.lnEmin; P.dlnE = s->tabs.dlnE;
  P.n_exc = s->tabs.n_exc;
  std::memcpy(P.exc, s->tabs.exc, sizeof(P.exc));
  P.Jr = s->Jr[0]; P.Jz = s->Jz[0];
  P.qEr = s->quads.er; P.qEz = s->quads.ez; P.qH = s->quads.h;
  {
    std::vector<double> iv(nr);
    for (int i = 0; i < nr; ++i) iv[i] = (1.0 / s->scale) / shell_volume(i, c.dr, c.dz, c.PHIp);
    std::vector<double> colc((size_t)3 * nr);
    fdtd_column_table(nr, fdtd_coef(s), iv.data(), c.flags, colc.data());
    if (cudaMemcpy(s->invV, iv.data(), (size_t)nr * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->fdtd_colc, colc.data(), (size_t)3 * nr * 8, cudaMemcpyHostToDevice) != cudaSuccess)
      return cleanup(fail(ctx, GASATT_E_CUDA, "volume table upload"));
  }
  if ((rc = sim_alloc(s, &s->d_P, 2)) || (rc = upload_params(s))) return cleanup(rc);
  if (fdtd_tile(c.fdtd_ratio) < 4)
    return cleanup(fail(ctx, GASATT_E_ARG, "fdtd_ratio too large for the fused field update (max 6)"));
  int dev = ctx->device, nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (c.fdtd_ratio == 1) {
    if ((rc = s->form == 0 ? setup_fdtd_tma<double>(s, nsm) : setup_fdtd_tma<float>(s, nsm)))
      return cleanup(rc);
  }
  int occ = 4;
  if (s->form == 0) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pass64, kBlock, 0);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pass32<0>, kBlock, 0);
  s->pass_grid = (unsigned)(nsm * (occ > 0 ? occ : 1));
  if (s->form == 1) {
    // FP32 blocks take chunks from a counter: no more blocks than chunks the
    // capacity can hold (small instances then leave the GPU to others)
    const long long chunks = (cap + P.chunk - 1) / P.chunk;
    if ((long long)s->pass_grid > chunks) s->pass_grid = (unsigned)(chunks > 0 ? chunks : 1);
  }
  // as many collision warps as fit on the device at once
  int occ_mcc = 1;
  if (s->form == 0) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_mcc, k_mcc64, kMccBlock, 0);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_mcc, k_collide32, kMccBlock, 0);
  s->mcc_grid = (unsigned)(nsm * (occ_mcc > 0 ? occ_mcc : 1));
  // zero state
  SimCounters z{};
  z.step = -1;
  z.cap = (unsigned long long)cap;
  if (cudaMemcpy(s->cnt, &z, sizeof(z), cudaMemcpyHostToDevice) != cudaSuccess)
    return cleanup(fail(ctx, GASATT_E_CUDA, "counter init"));
  for (int k = 0; k < 2; ++k) {
    cudaMemset(s->Er[k], 0, nfE * esz);
    cudaMemset(s->Ez[k], 0, nfZ * esz);
    cudaMemset(s->H[k], 0, nfH * esz);
  }
  for (int q = 0; q < 2; ++q) {
    cudaMemset(s->Jr[q], 0, ncur * 8);
    cudaMemset(s->Jz[q], 0, ncur * 8);
  }
  if (s->Jir) {
    cudaMemset(s->Jir, 0, ncur * 8);
    cudaMemset(s->Jiz, 0, ncur * 8);
  }
  for (int i = 0; i < 6; ++i)
    if (cudaEventCreate(&s->ev[i]) != cudaSuccess) return cleanup(fail(ctx, GASATT_E_CUDA, "event"));
  if (cudaEventCreateWithFlags(&s->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->join_ev, cudaEventDisableTiming) != cudaSuccess)
    return cleanup(fail(ctx, GASATT_E_CUDA, "event"));
  rc = build_graphs(s);
  if (rc) return cleanup(rc);
  if (cudaDeviceSynchronize() != cudaSuccess) return cleanup(fail(ctx, GASATT_E_CUDA, "sim init"));
  *out = s;
  return GASATT_OK;
}

int gasatt_sim_get_config(const gasatt_sim *s, gasatt_sim_config *cfg) {
  if (!s || !cfg) return GASATT_E_ARG;
  *cfg = s->cfg;
  return GASATT_OK;
}

int gasatt_sim_destroy(gasatt_sim *s) {
  if (!s) return GASATT_OK;
  cudaSetDevice(s->ctx->device);
  cudaDeviceSynchronize();
  drop_graphs(s);
  for (int i = 0; i < 6; ++i)
    if (s->ev[i]) cudaEventDestroy(s->ev[i]);
  if (s->fork_ev) cudaEventDestroy(s->fork_ev);
  if (s->join_ev) cudaEventDestroy(s->join_ev);
  for (void *p : s->allocs) cudaFree(p);
  if (s->h_cnt) cudaFreeHost(s->h_cnt);
  delete s;
  return GASATT_OK;
}

int gasatt_sim_load(gasatt_sim *s, const double *r, const double *z, const double *ur,
                    const double *ut, const double *uz, const uint64_t *id, int64_t n,
                    int on_device) {
  if (!s) return GASATT_E_ARG;
  gasatt_ctx *ctx = s->ctx;
  if (n < 0 || n > s->cfg.capacity) return fail(ctx, GASATT_E_CAPACITY, "load exceeds capacity");
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const double *src[5] = {r, z, ur, ut, uz};
  const double *d[5];
  const uint64_t *did = id;
  void *buf = nullptr;
  if (!on_device && n > 0) {
    int rc = scratch(ctx, (size_t)n * 48, &buf);
    if (rc) return rc;
    for (int i = 0; i < 5; ++i) {
      d[i] = (double *)buf + (size_t)i * n;
      GASATT_CUDA(ctx, cudaMemcpyAsync((void *)d[i], src[i], (size_t)n * 8, cudaMemcpyHostToDevice, st));
    }
    did = (uint64_t *)((double *)buf + 5 * (size_t)n);
    GASATT_CUDA(ctx, cudaMemcpyAsync((void *)did, id, (size_t)n * 8, cudaMemcpyHostToDevice, st));
  } else {
    for (int i = 0; i < 5; ++i) d[i] = src[i];
  }
  s->cur = 0;
  if (n > 0) {
    if (s->form == 0)
      k_load64<<<grid_for(n, kBlock), kBlock, 0, st>>>(s->s64[0], d[0], d[1], d[2], d[3], d[4], did, n);
    else
      k_load32<<<grid_for(n, kBlock), kBlock, 0, st>>>(s->s32[0], d[0], d[1], d[2], d[3], d[4], did, n,
                                                       s->cfg.n_r, s->cfg.n_z, s->cfg.dr, s->cfg.dz, s->cfg.c,
                                                       0);   // the first pass runs at step -1
    GASATT_LAUNCHED(ctx);
  }
  return sim_reset(s, n);
}

int gasatt_sim_set_gas_density(gasatt_sim *s, const double *density, int on_device) {
  if (!s) return GASATT_E_ARG;
  gasatt_ctx *ctx = s->ctx;
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t ncell = (size_t)s->cfg.n_r * s->cfg.n_z;
  std::vector<double> h;
  if (density) {
    h.resize(ncell);
    GASATT_CUDA(ctx, cudaMemcpy(h.data(), density, ncell * 8,
                                on_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost));
    for (double v : h)
      if (!(v >= 0) || !std::isfinite(v)) return fail(ctx, GASATT_E_ARG, "gas density: negative or not finite");
  }
  // collisions still queued were drawn against the old bound: apply them first
  SIM_TRY(flush_collisions(s));
  GASATT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  double n_max = s->cfg.gas_density;
  if (density) {
    if (!s->d_gas) {
      int rc = sim_alloc(s, &s->d_gas, ncell);
      if (rc) return rc;
    }
    GASATT_CUDA(ctx, cudaMemcpy(s->d_gas, h.data(), ncell * 8, cudaMemcpyHostToDevice));
    n_max = 0;
    for (double v : h) n_max = v > n_max ? v : n_max;
    s->P.gas = s->d_gas;
  } else {
    s->P.gas = nullptr;
  }
  set_collision_bound(s, n_max);
  SIM_TRY(upload_params(s));
  drop_graphs(s);                  // the step graphs hold the launch parameters
  return build_graphs(s);
}

int gasatt_sim_set_gas_temperature(gasatt_sim *s, const double *temperature, int on_device) {
  if (!s) return GASATT_E_ARG;
  gasatt_ctx *ctx = s->ctx;
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t ncell = (size_t)s->cfg.n_r * s->cfg.n_z;
  std::vector<double> h;
  if (temperature) {
    h.resize(ncell);
    GASATT_CUDA(ctx, cudaMemcpy(h.data(), temperature, ncell * 8,
                                on_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost));
    for (double &v : h) {
      if (!(v >= 0) || !std::isfinite(v))
        return fail(ctx, GASATT_E_ARG, "gas temperature: negative or not finite");
      v = std::sqrt(s->cfg.kb * v / s->cfg.m_ion);    // the spread the births use
    }
  }
  // ions of the collisions still queued are born at the old temperature
  SIM_TRY(flush_collisions(s));
  GASATT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (temperature) {
    if (!s->d_ion_sig) {
      int rc = sim_alloc(s, &s->d_ion_sig, ncell);
      if (rc) return rc;
    }
    GASATT_CUDA(ctx, cudaMemcpy(s->d_ion_sig, h.data(), ncell * 8, cudaMemcpyHostToDevice));
    s->P.ion_sig = s->d_ion_sig;
  } else {
    s->P.ion_sig = nullptr;
  }
  SIM_TRY(upload_params(s));
  drop_graphs(s);                  // the step graphs hold the launch parameters
  return build_graphs(s);
}

int gasatt_sim_birth_photo(gasatt_sim *s, int64_t n_photo, double photon_keV, double sigma_r,
                           uint64_t seed, uint64_t id_base) {
  if (!s) return GASATT_E_ARG;
  gasatt_ctx *ctx = s->ctx;
  if (n_photo < 0 || !(sigma_r > 0) || !(photon_keV * 1000 > kKShellEv))
    return fail(ctx, GASATT_E_ARG, "birth_photo: bad arguments");
  if (2 * n_photo > s->cfg.capacity) return fail(ctx, GASATT_E_CAPACITY, "birth_photo exceeds capacity");
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const auto &c = s->cfg;
  auto speed = [&](double E_ev) {                      // u = gamma v of kinetic energy E
    const double e = E_ev * c.q_e / (c.m_e * c.c * c.c);
    return c.c * std::sqrt(e * (2 + e));
  };
  const double Rp = c.n_r * c.dr, Lp = c.n_z * c.dz;
  const double r_max = std::nextafter(Rp, 0.0);
  s->cur = 0;
  if (n_photo > 0) {
    const unsigned g = grid_for(n_photo, kBlock);
    if (s->form == 0)
      k_birth_photo<0><<<g, kBlock, 0, st>>>(s->s64[0], s->s32[0], n_photo,
                                             speed(photon_keV * 1000 - kKShellEv), speed(kAugerEv),
                                             sigma_r, r_max, Lp, seed, id_base, c.n_r, c.n_z,
                                             c.dr, c.dz, c.c);
    else
      k_birth_photo<1><<<g, kBlock, 0, st>>>(s->s64[0], s->s32[0], n_photo,
                                             speed(photon_keV * 1000 - kKShellEv), speed(kAugerEv),
                                             sigma_r, r_max, Lp, seed, id_base, c.n_r, c.n_z,
                                             c.dr, c.dz, c.c);
    GASATT_LAUNCHED(ctx);
  }
  return sim_reset(s, 2 * n_photo);
}

int gasatt_sim_read(gasatt_sim *s, double *r, double *z, double *ur, double *ut, double *uz,
                    uint64_t *id, int64_t cap, int64_t *n_out, int on_device) {
  if (!s) return GASATT_E_ARG;
  gasatt_ctx *ctx = s->ctx;
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  SIM_TRY(flush_collisions(s));
  GASATT_CUDA(ctx, cudaMemcpyAsync(s->h_cnt, s->cnt, sizeof(SimCounters), cudaMemcpyDeviceToHost, st));
  GASATT_CUDA(ctx, cudaStreamSynchronize(st));
  const unsigned long long nt = s->h_cnt->n_total + s->h_cnt->n_births;
  const int64_t n = (int64_t)(nt < s->h_cnt->cap ? nt : s->h_cnt->cap);
  if (n_out) *n_out = n;
  if (n > cap) return fail(ctx, GASATT_E_CAPACITY, "read buffer too small");
  if (n == 0) return GASATT_OK;
  double *d[5] = {r, z, ur, ut, uz};
  uint64_t *did = id;
  void *buf = nullptr;
  if (!on_device) {
    int rc = scratch(ctx, (size_t)n * 48, &buf);
    if (rc) return rc;
    for (int i = 0; i < 5; ++i) d[i] = (double *)buf + (size_t)i * n;
    did = (uint64_t *)((double *)buf + 5 * (size_t)n);
  }
  if (s->form == 0)
    k_read64<<<grid_for(n, kBlock), kBlock, 0, st>>>(s->s64[s->cur], d[0], d[1], d[2], d[3], d[4], did, n);
  else
    k_read32<<<grid_for(n, kBlock), kBlock, 0, st>>>(s->s32[s->cur], d[0], d[1], d[2], d[3], d[4], did, n,
                                                     s->cfg.dr, s->cfg.dz, s->cfg.c);
  GASATT_LAUNCHED(ctx);
  if (!on_device) {
    double *h[5] = {r, z, ur, ut, uz};
    for (int i = 0; i < 5; ++i)
      GASATT_CUDA(ctx, cudaMemcpyAsync(h[i], d[i], (size_t)n * 8, cudaMemcpyDeviceToHost, st));
    GASATT_CUDA(ctx, cudaMemcpyAsync(id, did, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
  }
  GASATT_CUDA(ctx, cudaStreamSynchronize(st));
  return GASATT_OK;
}

int gasatt_sim_load_ions(gasatt_sim *s, const double *r, const double *z, const double *ur,
                         const double *ut, const double *uz, const uint64_t *id,
                         const int8_t *charge, int64_t n, int on_device) {
  if (!s) return GASATT_E_ARG;
  gasatt_ctx *ctx = s->ctx;
  if (s->cfg.ion_capacity <= 0) return fail(ctx, GASATT_E_STATE, "load_ions: no ion species (ion_capacity 0)");
  if (n < 0 || n > s->cfg.ion_capacity) return fail(ctx, GASATT_E_CAPACITY, "load_ions exceeds ion_capacity");
  if (n > 0 && (!r || !z || !ur || !ut || !uz || !id)) return fail(ctx, GASATT_E_ARG, "load_ions: null array");
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  SIM_TRY(flush_collisions(s));
  const double *src[5] = {r, z, ur, ut, uz};
  const double *d[5] = {r, z, ur, ut, uz};
  const uint64_t *did = id;
  const int8_t *dq = charge;
  if (!on_device && n > 0) {
    void *buf = nullptr;
    int rc = scratch(ctx, (size_t)n * 49, &buf);
    if (rc) return rc;
    for (int i = 0; i < 5; ++i) {
      d[i] = (double *)buf + (size_t)i * n;
      GASATT_CUDA(ctx, cudaMemcpyAsync((void *)d[i], src[i], (size_t)n * 8, cudaMemcpyHostToDevice, st));
    }
    did = (uint64_t *)((double *)buf + 5 * (size_t)n);
    GASATT_CUDA(ctx, cudaMemcpyAsync((void *)did, id, (size_t)n * 8, cudaMemcpyHostToDevice, st));
    if (charge) {
      dq = (int8_t *)(did + n);
      GASATT_CUDA(ctx, cudaMemcpyAsync((void *)dq, charge, (size_t)n, cudaMemcpyHostToDevice, st));
    }
  }
  if (n > 0) {
    k_ion_load<<<grid_for(n, kBlock), kBlock, 0, st>>>(s->P.ion, d[0], d[1], d[2], d[3], d[4], did, dq, n);
    GASATT_LAUNCHED(ctx);
  }
  const unsigned long long zc[3] = {(unsigned long long)n, 0ull, 0ull};   // n_ions, overflow, lost
  GASATT_CUDA(ctx, cudaMemcpyAsync((char *)s->cnt + offsetof(SimCounters, n_ions), zc, sizeof(zc),
                                   cudaMemcpyHostToDevice, st));
  GASATT_CUDA(ctx, cudaMemsetAsync(s->Jir, 0, jbytes(s), st));
  GASATT_CUDA(ctx, cudaMemsetAsync(s->Jiz, 0, jbytes(s), st));
  GASATT_CUDA(ctx, cudaStreamSynchronize(st));    // the host arrays zc and charge go out of scope
  return GASATT_OK;
}

int gasatt_sim_read_ions(gasatt_sim *s, double *r, double *z, double *ur, double *ut, double *uz,
                         uint64_t *id, int8_t *charge, int64_t cap, int64_t *n_out, int on_device) {
  if (!s) return GASATT_E_ARG;
  gasatt_ctx *ctx = s->ctx;
  if (s->cfg.ion_capacity <= 0) {
    if (n_out) *n_out = 0;
    return GASATT_OK;
  }
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  SIM_TRY(flush_collisions(s));
  GASATT_CUDA(ctx, cudaMemcpyAsync(s->h_cnt, s->cnt, sizeof(SimCounters), cudaMemcpyDeviceToHost, st));
  GASATT_CUDA(ctx, cudaStreamSynchronize(st));
  const unsigned long long nc = s->h_cnt->n_ions;
  const int64_t n = (int64_t)(nc < (unsigned long long)s->cfg.ion_capacity ? nc : s->cfg.ion_capacity);
  if (n_out) *n_out = n;
  if (n > cap) return fail(ctx, GASATT_E_CAPACITY, "read_ions buffer too small");
  if (n == 0) return GASATT_OK;
  if (!r || !z || !ur || !ut || !uz || !id || !charge) return fail(ctx, GASATT_E_ARG, "read_ions: null array");
  double *d[5] = {r, z, ur, ut, uz};
  uint64_t *did = id;
  int8_t *dq = charge;
  if (!on_device) {
    void *buf = nullptr;
    int rc = scratch(ctx, (size_t)n * 49, &buf);
    if (rc) return rc;
    for (int i = 0; i < 5; ++i) d[i] = (double *)buf + (size_t)i * n;
    did = (uint64_t *)((double *)buf + 5 * (size_t)n);
    dq = (int8_t *)(did + n);
  }
  k_ion_read<<<grid_for(n, kBlock), kBlock, 0, st>>>(s->P.ion, d[0], d[1], d[2], d[3], d[4], did, dq, n);
  GASATT_LAUNCHED(ctx);
  if (!on_device) {
    double *h[5] = {r, z, ur, ut, uz};
    for (int i = 0; i < 5; ++i)
      GASATT_CUDA(ctx, cudaMemcpyAsync(h[i], d[i], (size_t)n * 8, cudaMemcpyDeviceToHost, st));
    GASATT_CUDA(ctx, cudaMemcpyAsync(id, did, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
    GASATT_CUDA(ctx, cudaMemcpyAsync(charge, dq, (size_t)n, cudaMemcpyDeviceToHost, st));
  }
  GASATT_CUDA(ctx, cudaStreamSynchronize(st));
  return GASATT_OK;
}

namespace {
// the gather quads of whole float fields (after the fields are set from outside)
__global__ void k_build_quads(const float *Er, const float *Ez, const float *H, int nr, int nz,
                              int ld, FieldQuads q) {
  const int64_t nE = (int64_t)nr * (nz + 1), nZ = (int64_t)(nr + 1) * nz, nH = (int64_t)nr * nz;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nE + nZ + nH;
       k += (int64_t)gridDim.x * blockDim.x) {
    if (k < nE) {
      const int i = (int)(k % nr), j = (int)(k / nr);
      quad_put(q.er, nr + 1, quad_axis_shifted(i, nr), quad_axis_plain(j, nz), Er[i + (int64_t)j * ld]);
    } else if (k < nE + nZ) {
      const int64_t m = k - nE;
      const int i = (int)(m % (nr + 1)), j = (int)(m / (nr + 1));
      quad_put(q.ez, nr, quad_axis_plain(i, nr), quad_axis_shifted(j, nz), Ez[i + (int64_t)j * ld]);
    } else {
      const int64_t m = k - nE - nZ;
      const int i = (int)(m % nr), j = (int)(m / nr);
      quad_put(q.h, nr + 1, quad_axis_shifted(i, nr), quad_axis_shifted(j, nz), H[i + (int64_t)j * ld]);
    }
  }
}

// dense column-major double (ncol x nrow, the reference's layout) <-> the
// padded internal float layout (row stride ld)
__global__ void k_dense_to_strided(const double *src, float *dst, int ncol, int nrow, int ld) {
  const int64_t n = (int64_t)ncol * nrow;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(k % ncol), j = (int)(k / ncol);
    dst[i + (int64_t)j * ld] = (float)src[k];
  }
}
__global__ void k_strided_to_dense(const float *src, double *dst, int ncol, int nrow, int ld) {
  const int64_t n = (int64_t)ncol * nrow;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(k % ncol), j = (int)(k / ncol);
    dst[k] = (double)src[i + (int64_t)j * ld];
  }
}
__global__ void k_j_to_density(const unsigned long long *J, int nr, int nz, int ldj,
                               double inv_scale, double dr, double dz, double PHIp, double *out) {
  const int64_t n = (int64_t)nr * nz;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(k % nr), j = (int)(k / nr);
    out[k] = (double)(long long)J[i + (int64_t)j * ldj] * inv_scale / shell_volume(i, dr, dz, PHIp);
  }
}

int fields_io(gasatt_sim *s, double *Er, double *Ez, double *H, int on_device, bool set) {
  gasatt_ctx *ctx = s->ctx;
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int nr = s->cfg.n_r, nz = s->cfg.n_z, ld = s->ldf;
  const int ncol[3] = {nr, nr + 1, nr}, nrow[3] = {nz + 1, nz, nz};
  double *u[3] = {Er, Ez, H};
  void *dev[3] = {s->Er[fcur(s)], s->Ez[fcur(s)], s->H[fcur(s)]};
  if (s->form == 0) {
    // FP64: a pitched copy between the caller's dense array and the padded grid
    for (int f = 0; f < 3; ++f) {
      const size_t w = (size_t)ncol[f] * 8;
      if (set)
        GASATT_CUDA(ctx, cudaMemcpy2DAsync(dev[f], (size_t)ld * 8, u[f], w, w, nrow[f],
                                           on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
      else
        GASATT_CUDA(ctx, cudaMemcpy2DAsync(u[f], w, dev[f], (size_t)ld * 8, w, nrow[f],
                                           on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    }
    GASATT_CUDA(ctx, cudaStreamSynchronize(st));
    return GASATT_OK;
  }
  // FP32: through a dense double stage on the device when the caller's
  // arrays are host memory
  void *buf = nullptr;
  if (!on_device) {
    int rc = scratch(ctx, (size_t)((int64_t)ncol[0] * nrow[0] + (int64_t)ncol[1] * nrow[1] +
                                   (int64_t)ncol[2] * nrow[2]) * 8, &buf);
    if (rc) return rc;
  }
  int64_t off = 0;
  for (int f = 0; f < 3; ++f) {
    const int64_t n = (int64_t)ncol[f] * nrow[f];
    double *stage = on_device ? u[f] : (double *)buf + off;
    if (set) {
      if (!on_device) GASATT_CUDA(ctx, cudaMemcpyAsync(stage, u[f], n * 8, cudaMemcpyHostToDevice, st));
      k_dense_to_strided<<<grid_for(n, kBlock), kBlock, 0, st>>>(stage, (float *)dev[f], ncol[f], nrow[f], ld);
      GASATT_LAUNCHED(ctx);
    } else {
      k_strided_to_dense<<<grid_for(n, kBlock), kBlock, 0, st>>>((const float *)dev[f], stage, ncol[f], nrow[f], ld);
      GASATT_LAUNCHED(ctx);
      if (!on_device) GASATT_CUDA(ctx, cudaMemcpyAsync(u[f], stage, n * 8, cudaMemcpyDeviceToHost, st));
    }
    off += n;
  }
  if (set && s->quads.er) {
    const int64_t n = (int64_t)nr * (nz + 1) + (int64_t)(nr + 1) * nz + (int64_t)nr * nz;
    k_build_quads<<<grid_for(n, kBlock), kBlock, 0, st>>>(
        (const float *)s->Er[fcur(s)], (const float *)s->Ez[fcur(s)], (const float *)s->H[fcur(s)], nr, nz, ld,
        s->quads);
    GASATT_LAUNCHED(ctx);
  }
  GASATT_CUDA(ctx, cudaStreamSynchronize(st));
  return GASATT_OK;
}
}  // namespace

int gasatt_sim_set_fields(gasatt_sim *s, const double *Er, const double *Ez, const double *H,
                          int on_device) {
  if (!s) return GASATT_E_ARG;
  return fields_io(s, (double *)Er, (double *)Ez, (double *)H, on_device, true);
}

int gasatt_sim_get_fields(gasatt_sim *s, double *Er, double *Ez, double *H, int on_device) {
  if (!s) return GASATT_E_ARG;
  return fields_io(s, Er, Ez, H, on_device, false);
}

int gasatt_sim_get_current(gasatt_sim *s, double *jr, double *jz, int on_device) {
  if (!s) return GASATT_E_ARG;
  gasatt_ctx *ctx = s->ctx;
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int nr = s->cfg.n_r, nz = s->cfg.n_z;
  const int64_t n = (int64_t)nr * nz;
  double *d[2] = {jr, jz};
  void *buf = nullptr;
  if (!on_device) {
    int rc = scratch(ctx, (size_t)n * 16, &buf);
    if (rc) return rc;
    d[0] = (double *)buf; d[1] = (double *)buf + n;
  }
  const int q = (int)(s->host_step & 1);   // buffer of the most recent deposit
  const unsigned long long *J[2] = {s->Jr[q], s->Jz[q]};
  for (int f = 0; f < 2; ++f) {
    k_j_to_density<<<grid_for(n, kBlock), kBlock, 0, st>>>(J[f], nr, nz, s->ldj, 1.0 / s->scale,
                                                           s->cfg.dr, s->cfg.dz, s->cfg.PHIp, d[f]);
    GASATT_LAUNCHED(ctx);
  }
  if (!on_device) {
    GASATT_CUDA(ctx, cudaMemcpyAsync(jr, d[0], n * 8, cudaMemcpyDeviceToHost, st));
    GASATT_CUDA(ctx, cudaMemcpyAsync(jz, d[1], n * 8, cudaMemcpyDeviceToHost, st));
  }
  GASATT_CUDA(ctx, cudaStreamSynchronize(st));
  return GASATT_OK;
}

int gasatt_sim_sort(gasatt_sim *s) {
  if (!s) return GASATT_E_ARG;
  gasatt_ctx *ctx = s->ctx;
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  SIM_TRY(flush_collisions(s));            // the queue holds slot indices
  GASATT_CUDA(ctx, cudaGraphLaunch(s->g_sort[s->cur], ctx->stream));
  ctx->launches += 4;
  s->cur = 1 - s->cur;
  s->since_sort = 0;
  return GASATT_OK;
}

int gasatt_sim_step(gasatt_sim *s, int nsteps) {
  if (!s || nsteps < 0) return GASATT_E_ARG;
  gasatt_ctx *ctx = s->ctx;
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  SIM_TRY(sim_prime(s));
  // field update, (FP64: commit, collision kernel,) particle pass
  const int per_step = s->form == 0 ? 4 : 2;
  for (int k = 0; k < nsteps; ++k) {
    if (s->cfg.sort_period > 0 && s->since_sort >= s->cfg.sort_period) SIM_TRY(gasatt_sim_sort(s));
    GASATT_CUDA(ctx, cudaGraphLaunch(s->g_step[s->cur][s->host_step & 1], st));
    ctx->launches += per_step;
    s->host_step++;
    s->since_sort++;
    s->mcc_pending = true;
    if (ion_push_due(s)) SIM_TRY(launch_ion_push(s, st));
  }
  return GASATT_OK;
}

int gasatt_sim_diag(gasatt_sim *s, gasatt_diag *d) {
  if (!s || !d) return GASATT_E_ARG;
  gasatt_ctx *ctx = s->ctx;
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  SIM_TRY(flush_collisions(s));
  GASATT_CUDA(ctx, cudaMemsetAsync((char *)s->cnt + offsetof(SimCounters, kin_fx), 0, 16, st));
  if (s->form == 0) k_diag<0><<<s->pass_grid, kBlock, 0, st>>>(s->s64[s->cur], s->s32[s->cur], s->cnt, s->cfg.c, s->cfg.m_e, s->cfg.q_e);
  else k_diag<1><<<s->pass_grid, kBlock, 0, st>>>(s->s64[s->cur], s->s32[s->cur], s->cnt, s->cfg.c, s->cfg.m_e, s->cfg.q_e);
  GASATT_LAUNCHED(ctx);
  if (s->cfg.ion_capacity > 0) {
    GASATT_CUDA(ctx, cudaMemsetAsync((char *)s->cnt + offsetof(SimCounters, ion_alive), 0, 24, st));
    k_ion_diag<<<s->pass_grid, kBlock, 0, st>>>(s->P.ion, s->cfg.ion_capacity, s->cnt, s->cfg.c,
                                                  s->cfg.m_ion, s->cfg.q_e);
    GASATT_LAUNCHED(ctx);
  }
  const int nr = s->cfg.n_r, nz = s->cfg.n_z;
  if (s->form == 0)
    k_field_energy<double><<<s->partial_blocks, kBlock, 0, st>>>((double *)s->Er[fcur(s)], (double *)s->Ez[fcur(s)], (double *)s->H[fcur(s)], nr, nz, s->ldf, s->cfg.dr, s->cfg.dz, s->partial);
  else
    k_field_energy<float><<<s->partial_blocks, kBlock, 0, st>>>((float *)s->Er[fcur(s)], (float *)s->Ez[fcur(s)], (float *)s->H[fcur(s)], nr, nz, s->ldf, s->cfg.dr, s->cfg.dz, s->partial);
  GASATT_LAUNCHED(ctx);
  std::vector<double> part(2 * s->partial_blocks);
  GASATT_CUDA(ctx, cudaMemcpyAsync(s->h_cnt, s->cnt, sizeof(SimCounters), cudaMemcpyDeviceToHost, st));
  GASATT_CUDA(ctx, cudaMemcpyAsync(part.data(), s->partial, part.size() * 8, cudaMemcpyDeviceToHost, st));
  GASATT_CUDA(ctx, cudaStreamSynchronize(st));
  const SimCounters &h = *s->h_cnt;
  double we = 0, wm = 0;
  for (int b = 0; b < s->partial_blocks; ++b) { we += part[2 * b]; wm += part[2 * b + 1]; }
  d->n_alive = (int64_t)h.alive;
  d->n_total = (int64_t)(h.n_total + h.n_births < h.cap ? h.n_total + h.n_births : h.cap);
  d->n_ionizations = (int64_t)h.ion;
  d->n_elastic = (int64_t)h.ela;
  d->n_excitation = (int64_t)h.exc;
  d->n_null = (int64_t)h.nul;
  d->n_lost_wall = (int64_t)h.lost;
  d->n_ions = (int64_t)h.ion_alive;
  d->kinetic_ev = (double)h.kin_fx / 65536.0;
  d->field_energy_j = s->cfg.PHIp * 0.5 * s->cfg.eps0 * we + s->cfg.PHIp * 0.5 * s->cfg.mu0 * wm;
  d->steps = s->host_step;
  d->status_flags = (h.cap_overflow ? 2 : 0) | (h.ion_overflow ? 4 : 0) |
                    (h.fdtd_err || h.scan_err ? 8 : 0);
  d->n_ion_lost_wall = (int64_t)h.ion_lost;
  d->ion_kinetic_ev = (double)h.ion_kin_fx / 4294967296.0;
  d->net_charge_c = s->cfg.q_e * s->cfg.FN * ((double)h.ion_charge - (double)h.alive);
  d->collision_loss_ev = GASATT_ION_I_EV * (double)h.ion + (double)h.exc_loss_fx / 65536.0;
  d->wall_loss_ev = (double)h.wall_loss_fx / 65536.0;
  return GASATT_OK;
}

int gasatt_sim_counts(gasatt_sim *s, int64_t *n_slots, int64_t *n_ion, int64_t *n_lost) {
  if (!s) return GASATT_E_ARG;
  gasatt_ctx *ctx = s->ctx;
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  SIM_TRY(flush_collisions(s));
  GASATT_CUDA(ctx, cudaMemcpyAsync(s->h_cnt, s->cnt, sizeof(SimCounters), cudaMemcpyDeviceToHost, ctx->stream));
  GASATT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const SimCounters &h = *s->h_cnt;
  const unsigned long long nt = h.n_total + h.n_births;
  if (n_slots) *n_slots = (int64_t)(nt < h.cap ? nt : h.cap);
  if (n_ion) *n_ion = (int64_t)h.ion;
  if (n_lost) *n_lost = (int64_t)h.lost;
  return GASATT_OK;
}

int gasatt_sim_enable_timing(gasatt_sim *s, int enable) {
  if (!s) return GASATT_E_ARG;
  if ((bool)enable == s->timing) return GASATT_OK;
  GASATT_CUDA(s->ctx, cudaSetDevice(s->ctx->device));
  GASATT_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
  drop_graphs(s);
  s->timing = enable != 0;
  return build_graphs(s);
}

int gasatt_sim_last_timing(gasatt_sim *s, float *fdtd_ms, float *pass_ms, float *mcc_ms) {
  if (!s) return GASATT_E_ARG;
  if (!s->timing) return fail(s->ctx, GASATT_E_STATE, "timing not enabled");
  GASATT_CUDA(s->ctx, cudaEventSynchronize(s->ev[3]));
  float a = 0, b = 0, m = 0;
  GASATT_CUDA(s->ctx, cudaEventElapsedTime(&a, s->ev[0], s->ev[1]));
  if (s->form == 1) {
    // FP32: the pass runs the collisions itself; no separate collision kernel
    GASATT_CUDA(s->ctx, cudaEventElapsedTime(&b, s->ev[1], s->ev[3]));
  } else {
    GASATT_CUDA(s->ctx, cudaEventElapsedTime(&b, s->ev[2], s->ev[3]));
    GASATT_CUDA(s->ctx, cudaEventElapsedTime(&m, s->ev[4], s->ev[5]));
  }
  if (fdtd_ms) *fdtd_ms = a;
  if (pass_ms) *pass_ms = b;
  if (mcc_ms) *mcc_ms = m;
  return GASATT_OK;
}

}  // extern "C"

namespace {

// Cartesian (x, y, z, v) columns -> axisymmetric state (r, z, u = gamma v local), id = slot
__global__ void k_cart_in(const double *pos, const double *vel, int64_t ld, int64_t n, double c,
                          double *r, double *z, double *ur, double *ut, double *uz, uint64_t *id,
                          uint64_t id_base) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const double x = pos[p], y = pos[ld + p];
    const double vx = vel[p], vy = vel[ld + p], vz = vel[2 * ld + p];
    const double rr = sqrt(x * x + y * y);
    const double cp = rr > 0 ? x / rr : 1.0, sp = rr > 0 ? y / rr : 0.0;
    const double g = 1 / sqrt(1 - (vx * vx + vy * vy + vz * vz) / (c * c));
    r[p] = rr; z[p] = pos[2 * ld + p];
    ur[p] = g * (vx * cp + vy * sp); ut[p] = g * (-vx * sp + vy * cp); uz[p] = g * vz;
    id[p] = id_base + (uint64_t)p;
  }
}

// axisymmetric state -> Cartesian columns at azimuth 0, velocity v = u / gamma
__global__ void k_cart_out(const double *r, const double *z, const double *ur, const double *ut,
                           const double *uz, int64_t n, double c, double *pos, double *vel,
                           int64_t ld) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const double g = sqrt(1 + (ur[p] * ur[p] + ut[p] * ut[p] + uz[p] * uz[p]) / (c * c));
    pos[p] = r[p]; pos[ld + p] = 0.0; pos[2 * ld + p] = z[p];
    vel[p] = ur[p] / g; vel[ld + p] = ut[p] / g; vel[2 * ld + p] = uz[p] / g;
  }
}

}  // namespace

extern "C" {

int gasatt_sim_run_host(gasatt_sim *s, double *pos, double *vel, int64_t *n_io, int64_t cap,
                        int nsteps) {
  if (!s || !n_io || nsteps < 1) return GASATT_E_ARG;
  gasatt_ctx *ctx = s->ctx;
  const int64_t n = *n_io;
  if (n < 0 || n > cap || n > s->cfg.capacity) return fail(ctx, GASATT_E_ARG, "run_host: bad count");
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  // device staging: 6 columns in, reused for the way out; plus state scratch
  void *buf;
  const int64_t m = s->cfg.capacity;
  int rc = scratch(ctx, (size_t)m * 8 * 12, &buf);
  if (rc) return rc;
  double *dpos = (double *)buf, *dvel = dpos + 3 * m;
  double *sr = dvel + 3 * m, *sz = sr + m, *sur = sz + m, *sut = sur + m, *suz = sut + m;
  uint64_t *sid = (uint64_t *)(suz + m);
  for (int d = 0; d < 3; ++d) {
    GASATT_CUDA(ctx, cudaMemcpyAsync(dpos + d * m, pos + d * cap, (size_t)n * 8, cudaMemcpyHostToDevice, st));
    GASATT_CUDA(ctx, cudaMemcpyAsync(dvel + d * m, vel + d * cap, (size_t)n * 8, cudaMemcpyHostToDevice, st));
  }
  // the step counter keeps running across calls, so (id = slot, step) never repeats
  GASATT_CUDA(ctx, cudaMemcpyAsync(s->h_cnt, s->cnt, sizeof(SimCounters), cudaMemcpyDeviceToHost, st));
  GASATT_CUDA(ctx, cudaStreamSynchronize(st));
  if (n > 0) {
    k_cart_in<<<grid_for(n, kBlock), kBlock, 0, st>>>(dpos, dvel, m, n, s->cfg.c, sr, sz, sur, sut, suz, sid, 0);
    GASATT_LAUNCHED(ctx);
    if (s->form == 0)
      k_load64<<<grid_for(n, kBlock), kBlock, 0, st>>>(s->s64[s->cur], sr, sz, sur, sut, suz, sid, n);
    else
      k_load32<<<grid_for(n, kBlock), kBlock, 0, st>>>(s->s32[s->cur], sr, sz, sur, sut, suz, sid, n,
                                                       s->cfg.n_r, s->cfg.n_z, s->cfg.dr, s->cfg.dz, s->cfg.c,
                                                       (int)(((s->h_cnt->step + 1) & 1) ^ 1));
    GASATT_LAUNCHED(ctx);
  }
  SimCounters h = *s->h_cnt;
  h.n_total = (unsigned long long)n;
  h.n_births = 0;
  h.n_cand[0] = h.n_cand[1] = 0;
  h.uncommitted = 0;
  h.chunk_next = 0;
  h.step += 1;                               // never reuse the last pass's step
  GASATT_CUDA(ctx, cudaMemcpyAsync(s->cnt, &h, sizeof(h), cudaMemcpyHostToDevice, st));
  for (int q = 0; q < 2; ++q) {
    GASATT_CUDA(ctx, cudaMemsetAsync(s->Jr[q], 0, jbytes(s), st));
    GASATT_CUDA(ctx, cudaMemsetAsync(s->Jz[q], 0, jbytes(s), st));
  }
  s->primed = false;
  s->mcc_pending = false;
  SIM_TRY(restart_steps(s, st));             // the prologue deposits into buffer 0
  s->since_sort = s->cfg.sort_period;       // sort the fresh population first
  SIM_TRY(gasatt_sim_step(s, nsteps - 1));
  // last step: the pending collisions, the fields, then a push that ends at
  // integer time
  SIM_TRY(flush_collisions(s));
  SIM_TRY(launch_fdtd(s, st, (int)(s->host_step & 1)));
  SIM_TRY(launch_pass(s, st, 2, (int)((s->host_step + 1) & 1), (int)(s->host_step & 1),
                      (int)((s->host_step + 1) & 1)));
  if (s->form == 0) SIM_TRY(launch_commit(s, st, (int)(s->host_step & 1)));
  SIM_TRY(gasatt_sim_sort(s));               // compacts away the dead
  s->host_step++;
  s->primed = false;
  GASATT_CUDA(ctx, cudaMemcpyAsync(s->h_cnt, s->cnt, sizeof(SimCounters), cudaMemcpyDeviceToHost, st));
  GASATT_CUDA(ctx, cudaStreamSynchronize(st));
  const int64_t nout = (int64_t)s->h_cnt->n_total;
  const int64_t nw = nout < cap ? nout : cap;
  if (nw > 0) {
    if (s->form == 0)
      k_read64<<<grid_for(nw, kBlock), kBlock, 0, st>>>(s->s64[s->cur], sr, sz, sur, sut, suz, sid, nw);
    else
      k_read32<<<grid_for(nw, kBlock), kBlock, 0, st>>>(s->s32[s->cur], sr, sz, sur, sut, suz, sid, nw,
                                                        s->cfg.dr, s->cfg.dz, s->cfg.c);
    GASATT_LAUNCHED(ctx);
    k_cart_out<<<grid_for(nw, kBlock), kBlock, 0, st>>>(sr, sz, sur, sut, suz, nw, s->cfg.c, dpos, dvel, m);
    GASATT_LAUNCHED(ctx);
    for (int d = 0; d < 3; ++d) {
      GASATT_CUDA(ctx, cudaMemcpyAsync(pos + d * cap, dpos + d * m, (size_t)nw * 8, cudaMemcpyDeviceToHost, st));
      GASATT_CUDA(ctx, cudaMemcpyAsync(vel + d * cap, dvel + d * m, (size_t)nw * 8, cudaMemcpyDeviceToHost, st));
    }
  }
  GASATT_CUDA(ctx, cudaStreamSynchronize(st));
  *n_io = nw;
  if (nout > cap) return fail(ctx, GASATT_E_CAPACITY, "run_host: more electrons than cap rows");
  return GASATT_OK;
}

// ================================================================ batches
// Many independent gas cells stepped together.  Cells of the same precision
// form and field patch (fdtd_ratio 1) form a group that runs each step as a
// few launches for the whole group - the field update over every cell's
// tiles (k_batch_fdtd_tma), (FP64: the commits and the collisions beside it,)
// then the particle pass over every cell's candidates and chunks
// (k_batch_pass32 / k_batch_pass64) - instead of one set of launches per
// cell, so the blocks of each launch share all cells' work and small cells
// do not leave the GPU idle.  Groups, and any cell that fits no group
// (fdtd_ratio > 1), run side by side as branches of one graph.  The cells
// share a sort period, so they swap state buffers in lockstep; if one is
// ever out of step (stepped on its own in between), the batch steps each
// cell with its own graph.
struct BatchGroup {
  int form = 0, ph = 0;
  std::vector<gasatt_sim *> sims;
  void *cells = nullptr;                 // BatchCell32 / BatchCell64 per cell
  FdtdInst *insts[2] = {nullptr, nullptr};   // per step parity (the current buffer read)
  int2 *table = nullptr;                 // (cell, tile) work items of the field update
  int nitems = 0;
  SimCounters **commit = nullptr;        // FP32: counters the field update commits
  unsigned long long *chunk_next = nullptr;
  unsigned fdtd_grid = 0, pass_grid = 0, mcc_grid = 0;
  size_t fdtd_smem = 0;
};

struct gasatt_batch {
  gasatt_ctx *ctx = nullptr;
  std::vector<gasatt_sim *> sims;
  std::vector<BatchGroup> groups;
  std::vector<gasatt_sim *> singles;     // cells stepped by their own step graph
  std::vector<void *> allocs;
  int sort_period = 0;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  cudaGraphExec_t g[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [state buffer][parity]
  cudaGraphExec_t g_sort[2] = {nullptr, nullptr};   // every cell's sort side by side [state buffer]
};

int gasatt_batch_destroy(gasatt_batch *b) {
  if (!b) return GASATT_OK;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  for (int i = 0; i < 2; ++i) {
    for (int q = 0; q < 2; ++q)
      if (b->g[i][q]) cudaGraphExecDestroy(b->g[i][q]);
    if (b->g_sort[i]) cudaGraphExecDestroy(b->g_sort[i]);
  }
  if (b->fork_ev) cudaEventDestroy(b->fork_ev);
  if (b->join_ev) cudaEventDestroy(b->join_ev);
  for (void *p : b->allocs) cudaFree(p);
  delete b;
  return GASATT_OK;
}

extern "C++" {
namespace {

template <typename T>
int batch_alloc(gasatt_batch *b, T **p, size_t n) {
  cudaError_t e = cudaMalloc((void **)p, (n ? n : 1) * sizeof(T));
  if (e != cudaSuccess) return cuda_fail(b->ctx, e, "cudaMalloc (batch)");
  b->allocs.push_back((void *)*p);
  return GASATT_OK;
}

// device tables of a group: the cells' pass and field-update descriptors,
// the field update's work items, the commit list, the chunk counter, grids
int batch_group_setup(gasatt_batch *b, BatchGroup &G) {
  gasatt_ctx *ctx = b->ctx;
  const int n = (int)G.sims.size();
  if (G.form == 1) {
    std::vector<BatchCell32> h(n);
    std::vector<SimCounters *> cm(n);
    for (int i = 0; i < n; ++i) {
      gasatt_sim *s = G.sims[i];
      for (int jb = 0; jb < 2; ++jb) {
        h[i].P[jb] = s->P;
        h[i].P[jb].Jr = s->Jr[jb]; h[i].P[jb].Jz = s->Jz[jb];
      }
      h[i].S[0] = s->s32[0]; h[i].S[1] = s->s32[1];
      h[i].cnt = s->cnt; h[i].queue = s->queue;
      for (int k = 0; k < 2; ++k) h[i].F[k] = Fields<float>{(float *)s->Er[k], (float *)s->Ez[k], (float *)s->H[k]};
      cm[i] = s->cnt;
    }
    BatchCell32 *d;
    SIM_TRY(batch_alloc(b, &d, (size_t)n));
    GASATT_CUDA(ctx, cudaMemcpy(d, h.data(), sizeof(BatchCell32) * n, cudaMemcpyHostToDevice));
    G.cells = d;
    SIM_TRY(batch_alloc(b, &G.commit, (size_t)n));
    GASATT_CUDA(ctx, cudaMemcpy(G.commit, cm.data(), sizeof(SimCounters *) * n, cudaMemcpyHostToDevice));
  } else {
    std::vector<BatchCell64> h(n);
    for (int i = 0; i < n; ++i) {
      gasatt_sim *s = G.sims[i];
      for (int jb = 0; jb < 2; ++jb) {
        h[i].P[jb] = s->P;
        h[i].P[jb].Jr = s->Jr[jb]; h[i].P[jb].Jz = s->Jz[jb];
      }
      h[i].S[0] = s->s64[0]; h[i].S[1] = s->s64[1];
      h[i].cnt = s->cnt; h[i].queue = s->queue;
      for (int k = 0; k < 2; ++k) h[i].F[k] = Fields<double>{(double *)s->Er[k], (double *)s->Ez[k], (double *)s->H[k]};
    }
    BatchCell64 *d;
    SIM_TRY(batch_alloc(b, &d, (size_t)n));
    GASATT_CUDA(ctx, cudaMemcpy(d, h.data(), sizeof(BatchCell64) * n, cudaMemcpyHostToDevice));
    G.cells = d;
  }
  std::vector<int2> table;
  for (int i = 0; i < n; ++i)
    for (int t = 0; t < G.sims[i]->fdtd_inst[0].ntiles; ++t) table.push_back(make_int2(i, t));
  G.nitems = (int)table.size();
  SIM_TRY(batch_alloc(b, &G.table, table.size()));
  GASATT_CUDA(ctx, cudaMemcpy(G.table, table.data(), sizeof(int2) * table.size(), cudaMemcpyHostToDevice));
  for (int q = 0; q < 2; ++q) {
    std::vector<FdtdInst> hi(n);
    for (int i = 0; i < n; ++i) hi[i] = G.sims[i]->fdtd_inst[q];
    SIM_TRY(batch_alloc(b, &G.insts[q], (size_t)n));
    GASATT_CUDA(ctx, cudaMemcpy(G.insts[q], hi.data(), sizeof(FdtdInst) * n, cudaMemcpyHostToDevice));
  }
  SIM_TRY(batch_alloc(b, &G.chunk_next, 1));
  int nsm = 148, occ = 1;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
  G.fdtd_smem = G.sims[0]->tma_smem;
  const BatchFdtdTmaFn fk = G.form == 1 ? batch_fdtd_tma_fn<float>(G.ph) : batch_fdtd_tma_fn<double>(G.ph);
  GASATT_CUDA(ctx, cudaFuncSetAttribute(fk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G.fdtd_smem));
  GASATT_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fk, 32 * kTmaWarps, G.fdtd_smem));
  const long long fslots = (long long)nsm * (occ > 0 ? occ : 1);
  const long long fblocks = (G.nitems + kTmaWarps - 1) / kTmaWarps;
  G.fdtd_grid = (unsigned)(fslots < fblocks ? fslots : (fblocks > 0 ? fblocks : 1));
  occ = 1;
  if (G.form == 1) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch_pass32, kBlock, 0);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch_pass64, kBlock, 0);
  G.pass_grid = (unsigned)(nsm * (occ > 0 ? occ : 1));
  occ = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch_mcc64, kMccBlock, 0);
  G.mcc_grid = (unsigned)(nsm * (occ > 0 ? occ : 1));
  return GASATT_OK;
}

// one step of group G (state buffer cur, step parity q) onto the capturing
// stream cs (side: a second stream for the FP64 collision branch)
int batch_group_launch(gasatt_batch *b, BatchGroup &G, cudaStream_t cs, cudaStream_t side, int cur,
                       int q) {
  gasatt_ctx *ctx = b->ctx;
  const int n = (int)G.sims.size();
  const dim3 fb(32 * kTmaWarps);
  if (G.form == 1) {
    batch_fdtd_tma_fn<float>(G.ph)<<<G.fdtd_grid, fb, G.fdtd_smem, cs>>>(G.insts[q], G.table, G.nitems,
                                                                        G.commit, n);
    GASATT_CUDA(ctx, cudaGetLastError());
    GASATT_CUDA(ctx, cudaMemsetAsync(G.chunk_next, 0, 8, cs));
    k_batch_pass32<<<G.pass_grid, kBlock, 0, cs>>>((const BatchCell32 *)G.cells, n, cur, 1 - q,
                                                   G.chunk_next);
    GASATT_CUDA(ctx, cudaGetLastError());
    return GASATT_OK;
  }
  GASATT_CUDA(ctx, cudaEventRecord(b->fork_ev, cs));
  GASATT_CUDA(ctx, cudaStreamWaitEvent(side, b->fork_ev, 0));
  k_batch_commit64<<<1, 256, 0, side>>>((const BatchCell64 *)G.cells, n, 1 - q);
  k_batch_mcc64<<<G.mcc_grid, kMccBlock, 0, side>>>((const BatchCell64 *)G.cells, n, cur, 1 - q);
  GASATT_CUDA(ctx, cudaGetLastError());
  GASATT_CUDA(ctx, cudaEventRecord(b->join_ev, side));
  batch_fdtd_tma_fn<double>(G.ph)<<<G.fdtd_grid, fb, G.fdtd_smem, cs>>>(G.insts[q], G.table, G.nitems,
                                                                       nullptr, n);
  GASATT_CUDA(ctx, cudaGetLastError());
  GASATT_CUDA(ctx, cudaStreamWaitEvent(cs, b->join_ev, 0));
  GASATT_CUDA(ctx, cudaMemsetAsync(G.chunk_next, 0, 8, cs));
  k_batch_pass64<<<G.pass_grid, kBlock, 0, cs>>>((const BatchCell64 *)G.cells, n, cur, 1 - q, 0, q,
                                                 G.chunk_next);
  GASATT_CUDA(ctx, cudaGetLastError());
  return GASATT_OK;
}

int batch_build_graphs(gasatt_batch *b) {
  gasatt_ctx *ctx = b->ctx;
  cudaStream_t cs, side;
  GASATT_CUDA(ctx, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  if (cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking) != cudaSuccess) {
    cudaStreamDestroy(cs);
    return fail(ctx, GASATT_E_CUDA, "batch: stream");
  }
  int rc = GASATT_OK;
  for (int bi = 0; bi < 2 && !rc; ++bi) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) { rc = cuda_fail(ctx, e, "batch sort graph"); break; }
    for (size_t i = 0; i < b->sims.size() && !rc; ++i) {
      cudaGraphNode_t node;
      e = cudaGraphAddChildGraphNode(&node, g, nullptr, 0, b->sims[i]->gr_sort[bi]);
      if (e != cudaSuccess) rc = cuda_fail(ctx, e, "batch sort graph");
    }
    if (!rc) {
      e = cudaGraphInstantiate(&b->g_sort[bi], g, 0);
      if (e != cudaSuccess) rc = cuda_fail(ctx, e, "batch sort graph");
    }
    cudaGraphDestroy(g);
  }
  for (int bi = 0; bi < 2 && !rc; ++bi)
    for (int q = 0; q < 2 && !rc; ++q) {
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaGraphCreate(&g, 0);
      if (e != cudaSuccess) { rc = cuda_fail(ctx, e, "batch graph"); break; }
      for (BatchGroup &G : b->groups) {
        cudaGraph_t child = nullptr;
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) { rc = cuda_fail(ctx, e, "batch capture"); break; }
        rc = batch_group_launch(b, G, cs, side, bi, q);
        const cudaError_t e2 = cudaStreamEndCapture(cs, &child);
        if (!rc && e2 != cudaSuccess) rc = cuda_fail(ctx, e2, "batch capture");
        if (!rc) {
          cudaGraphNode_t node;
          e = cudaGraphAddChildGraphNode(&node, g, nullptr, 0, child);
          if (e != cudaSuccess) rc = cuda_fail(ctx, e, "batch graph");
        }
        if (child) cudaGraphDestroy(child);
        if (rc) break;
      }
      for (size_t i = 0; i < b->singles.size() && !rc; ++i) {
        cudaGraphNode_t node;
        e = cudaGraphAddChildGraphNode(&node, g, nullptr, 0, b->singles[i]->gr_step[bi][q]);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "batch graph");
      }
      if (!rc) {
        e = cudaGraphInstantiate(&b->g[bi][q], g, 0);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "batch graph");
      }
      cudaGraphDestroy(g);
    }
  cudaStreamDestroy(side);
  cudaStreamDestroy(cs);
  return rc;
}

// flush_collisions for every cell of the batch (before its sort): a group
// whose cells are at the same step parity and state buffer does it in two
// launches (FP32: k_batch_collide32) or three (FP64: the commits, then
// k_batch_mcc64) for all of its cells, then empties their queues; any other
// cell flushes on its own.  A cell with nothing pending finds an empty queue
// (its own flush emptied it) and a commit already made.
int batch_flush_collisions(gasatt_batch *b) {
  gasatt_ctx *ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  for (BatchGroup &G : b->groups) {
    const gasatt_sim *s0 = G.sims[0];
    bool same = true, any = false;
    for (const gasatt_sim *s : G.sims) {
      same = same && s->cur == s0->cur && (s->host_step & 1) == (s0->host_step & 1);
      any = any || s->mcc_pending;
    }
    if (!any) continue;
    if (!same) {
      for (gasatt_sim *s : G.sims) SIM_TRY(flush_collisions(s));
      continue;
    }
    const int n = (int)G.sims.size(), cur = s0->cur, q = (int)((s0->host_step - 1) & 1);
    if (G.form == 1) {
      k_batch_collide32<<<G.pass_grid, kMccBlock, 0, st>>>((const BatchCell32 *)G.cells, n, cur);
      k_batch_clear_cand<<<1, 256, 0, st>>>((const BatchCell32 *)G.cells, n, q);
      ctx->launches += 2;
    } else {
      k_batch_commit64<<<1, 256, 0, st>>>((const BatchCell64 *)G.cells, n, q);
      k_batch_mcc64<<<G.mcc_grid, kMccBlock, 0, st>>>((const BatchCell64 *)G.cells, n, cur, q);
      k_batch_clear_cand<<<1, 256, 0, st>>>((const BatchCell64 *)G.cells, n, q);
      ctx->launches += 3;
    }
    GASATT_CUDA(ctx, cudaGetLastError());
    for (gasatt_sim *s : G.sims) s->mcc_pending = false;
  }
  for (gasatt_sim *s : b->singles) SIM_TRY(flush_collisions(s));
  return GASATT_OK;
}

}  // namespace
}  // extern "C++"

int gasatt_batch_create(gasatt_ctx *ctx, gasatt_sim *const *sims, int n, int sort_period,
                        gasatt_batch **out) {
  if (!ctx || !sims || n < 1 || !out || sort_period < 0)
    return fail(ctx, GASATT_E_ARG, "batch: bad arguments");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (!sims[i] || sims[i]->ctx != ctx)
      return fail(ctx, GASATT_E_ARG, "batch: every instance must belong to this context");
    if (sims[i]->timing) return fail(ctx, GASATT_E_STATE, "batch: disable phase timing first");
    for (int j = 0; j < i; ++j)
      if (sims[j] == sims[i]) return fail(ctx, GASATT_E_ARG, "batch: an instance appears twice");
  }
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  gasatt_batch *b = new gasatt_batch();
  b->ctx = ctx;
  b->sims.assign(sims, sims + n);
  b->sort_period = sort_period;
  for (gasatt_sim *s : b->sims) s->cfg.sort_period = sort_period;
  // groups of cells with the same form and field patch; up to kMaxBatch each
  for (gasatt_sim *s : b->sims) {
    if (s->cfg.fdtd_ratio != 1) { b->singles.push_back(s); continue; }
    BatchGroup *G = nullptr;
    for (BatchGroup &g : b->groups)
      if (g.form == s->form && g.ph == s->tma_rows && (int)g.sims.size() < kMaxBatch) G = &g;
    if (!G) {
      b->groups.emplace_back();
      G = &b->groups.back();
      G->form = s->form;
      G->ph = s->tma_rows;
    }
    G->sims.push_back(s);
  }
  int rc = GASATT_OK;
  if (cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->join_ev, cudaEventDisableTiming) != cudaSuccess)
    rc = fail(ctx, GASATT_E_CUDA, "batch: event");
  for (size_t i = 0; i < b->groups.size() && !rc; ++i) rc = batch_group_setup(b, b->groups[i]);
  if (!rc) rc = batch_build_graphs(b);
  if (rc) {
    gasatt_batch_destroy(b);
    return rc;
  }
  *out = b;
  return GASATT_OK;
}

int gasatt_batch_step(gasatt_batch *b, int nsteps) {
  if (!b || nsteps < 0) return GASATT_E_ARG;
  gasatt_ctx *ctx = b->ctx;
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  for (int k = 0; k < nsteps; ++k) {
    for (gasatt_sim *s : b->sims) SIM_TRY(sim_prime(s));
    if (b->sort_period > 0) {
      // every cell due at once (the batch keeps them in lockstep): one graph
      // sorts them all side by side
      bool all_due = true;
      for (const gasatt_sim *s : b->sims)
        all_due = all_due && s->since_sort >= b->sort_period && s->cur == b->sims[0]->cur;
      if (all_due) {
        SIM_TRY(batch_flush_collisions(b));
        GASATT_CUDA(ctx, cudaGraphLaunch(b->g_sort[b->sims[0]->cur], st));
        for (gasatt_sim *s : b->sims) {
          ctx->launches += 4;
          s->cur = 1 - s->cur;
          s->since_sort = 0;
        }
      } else {
        for (gasatt_sim *s : b->sims)
          if (s->since_sort >= b->sort_period) SIM_TRY(gasatt_sim_sort(s));
      }
    }
    const gasatt_sim *s0 = b->sims[0];
    bool lockstep = true;
    for (const gasatt_sim *s : b->sims)
      lockstep = lockstep && s->cur == s0->cur && (s->host_step & 1) == (s0->host_step & 1) &&
                 !s->timing;
    if (lockstep) {
      GASATT_CUDA(ctx, cudaGraphLaunch(b->g[s0->cur][s0->host_step & 1], st));
      for (const BatchGroup &G : b->groups) ctx->launches += G.form == 0 ? 4 : 2;
      for (const gasatt_sim *s : b->singles) ctx->launches += s->form == 0 ? 4 : 2;
    } else {
      for (gasatt_sim *s : b->sims) {
        GASATT_CUDA(ctx, cudaGraphLaunch(s->g_step[s->cur][s->host_step & 1], st));
        ctx->launches += s->form == 0 ? 4 : 2;
      }
    }
    for (gasatt_sim *s : b->sims) {
      s->host_step++;
      s->since_sort++;
      s->mcc_pending = true;
      if (ion_push_due(s)) SIM_TRY(launch_ion_push(s, st));
    }
  }
  return GASATT_OK;
}

}  // extern "C"
