// tables.cpp - host construction of the N2 cross-section tables.
//
//  * find_cs0_host: find_CS0.m:1-61 on one energy (interp1 restated as
//    linear interpolation that is NaN outside the knots).
//  * build_elastic_tables: electron_collision.m:12-33 (combined TCS, log
//    energies and log DCS of the 36 DCS columns).
//  * build_sim_tables: the resident simulation's tables - sigma on G
//    log-spaced energies, per-energy normalised elastic CDFs (the
//    get_ElasticSc_sub1.m recipe: log DCS linear in log E, PDF = 2 pi sin
//    theta DCS, trapezoid CDF), and the FP64 null-collision bound.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include "gasatt_internal.h"

namespace gasatt {

namespace {

double interp1(const double *x, int sx, const double *y, int sy, int n, double xq) {
  if (!(xq >= x[0] && xq <= x[(int64_t)(n - 1) * sx])) return NAN;
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (x[(int64_t)mid * sx] <= xq) lo = mid; else hi = mid;
  }
  const double x0 = x[(int64_t)lo * sx], x1 = x[(int64_t)hi * sx];
  const double y0 = y[(int64_t)lo * sy], y1 = y[(int64_t)hi * sy];
  return y0 + (xq - x0) * (y1 - y0) / (x1 - x0);
}

// power-law continuation through the last two knots
double loglog_tail(const double *x, int sx, const double *y, int sy, int n, double xq) {
  const double x0 = x[(int64_t)(n - 2) * sx], x1 = x[(int64_t)(n - 1) * sx];
  const double y0 = y[(int64_t)(n - 2) * sy], y1 = y[(int64_t)(n - 1) * sy];
  const double s = std::log(y1 / y0) / std::log(x1 / x0);
  return y1 * std::pow(xq / x1, s);
}

}  // namespace

int check_tables(const gasatt_tables *t, std::string &err) {
  if (!t || !t->t_el || !t->t_sel || !t->t_sel_1 || !t->t_del || !t->t_sdel || !t->t_ion ||
      !t->t_exc) {
    err = "cross-section table pointer is NULL";
    return GASATT_E_TABLES;
  }
  if (t->n_el < 2 || t->n_sel < 2 || t->n_sel1 < 2 || t->n_ion < 2 || t->n_exc < 1 ||
      t->n_exc > 16) {
    err = "cross-section table too short";
    return GASATT_E_TABLES;
  }
  if (t->del_rows != 182 || t->sdel_rows != 182) {
    err = "DCS tables must have 182 rows (energy row + 181 angles)";
    return GASATT_E_TABLES;
  }
  if ((t->sdel_cols - 1) + (t->del_cols - 1) != (t->n_sel1 - 1) + t->n_el) {
    err = "DCS energy columns do not match the combined TCS rows";
    return GASATT_E_TABLES;
  }
  return GASATT_OK;
}

void find_cs0_host(const gasatt_tables *t, double E, double &se, double &si, double &sx,
                   unsigned flags) {
  const bool faithful = (flags & GASATT_Q_XS_NAN) != 0;
  const double *t_el = t->t_el, *t_sel = t->t_sel, *t_ion = t->t_ion, *t_exc = t->t_exc;
  const int n_el = t->n_el, n_sel = t->n_sel, n_ion = t->n_ion, n_exc = t->n_exc;
  double sel = 0.0;
  if (E >= 0.05) {                                     // find_CS0.m:102-107
    sel = interp1(&t_el[0], 2, &t_el[1], 2, n_el, E);
    if (!faithful && E > t_el[2 * (n_el - 1)]) sel = loglog_tail(&t_el[0], 2, &t_el[1], 2, n_el, E);
    sel = sel * GASATT_A0SQ * 2;
  } else if (E < 0.05) {                               // find_CS0.m:108-111
    double Ev = E * 1000;
    if (!faithful && Ev < t_sel[0]) Ev = t_sel[0];
    sel = interp1(&t_sel[0], 1, &t_sel[n_sel], 1, n_sel, Ev) * 1e-20;
  }
  se = sel;
  const double T = E * 1000;                           // find_CS0.m:116-119
  if (!faithful && T <= t_ion[0]) si = 0.0;
  else if (!faithful && T > t_ion[n_ion - 1])
    si = loglog_tail(&t_ion[0], 1, &t_ion[n_ion], 1, n_ion, T) * 1e-20;
  else si = interp1(&t_ion[0], 1, &t_ion[n_ion], 1, n_ion, T) * 1e-20;
  double s = 0.0;                                      // find_CS0.m:123-142
  for (int i = 0; i < n_exc; ++i) {
    const double k = t_exc[i], A = t_exc[n_exc + i], om = t_exc[2 * n_exc + i];
    const double nu = t_exc[3 * n_exc + i], ga = t_exc[4 * n_exc + i];
    if (!faithful && !(T > k)) continue;
    const double a = GASATT_CS_Q0 * A / (k * k);
    const double b = std::pow(k / T, om);
    const double c = std::pow(1 - std::pow(k / T, ga), nu);
    s = s + a * b * c;
  }
  sx = s * 1e-4;
}

int build_elastic_tables(const gasatt_tables *t, ElasticTables &o, std::string &err) {
  int st = check_tables(t, err);
  if (st) return st;
  const int m1 = t->n_sel1 - 1;                        // drop the 50 eV row (:17)
  o.ne = m1 + t->n_el;
  o.xInterp.assign(o.ne, 0.0);
  o.yInterp.assign(o.ne, 0.0);
  o.V.assign((size_t)o.ne * 181, 0.0);
  for (int i = 0; i < m1; ++i)                          // :15 a0^2 per N atom
    o.yInterp[i] = t->t_sel_1[t->n_sel1 + i] * 1e-20 / GASATT_A0SQ / 2;
  for (int i = 0; i < t->n_el; ++i) o.yInterp[m1 + i] = t->t_el[2 * i + 1];
  int col = 0;                                          // [t_sdel, t_del(:,2:end)]
  auto take = [&](const double *tab, int cols) {
    for (int c = 1; c < cols; ++c, ++col) {
      o.xInterp[col] = std::log(tab[(int64_t)c * 182]);
      for (int k = 0; k < 181; ++k)
        o.V[(size_t)col * 181 + k] = std::log(tab[(int64_t)c * 182 + 1 + k]);
    }
  };
  take(t->t_sdel, t->sdel_cols);
  take(t->t_del, t->del_cols);
  return GASATT_OK;
}

int build_sim_tables(const gasatt_tables *t, int G, double emin_ev, double emax_ev, double n_gas,
                     double c, double me, double qe, SimTables &o, std::string &err) {
  ElasticTables el;
  int st = build_elastic_tables(t, el, err);
  if (st) return st;
  if (G < 2 || !(emin_ev > 0) || !(emax_ev > emin_ev)) {
    err = "bad energy grid";
    return GASATT_E_ARG;
  }
  o.G = G;
  o.lnEmin = std::log(emin_ev);
  o.dlnE = (std::log(emax_ev) - o.lnEmin) / (G - 1);
  o.sig_el.assign(G, 0.0); o.sig_ion.assign(G, 0.0); o.sig_exc.assign(G, 0.0);
  o.edep.assign(G, 0.0);
  o.cdf.assign((size_t)G * 181, 0.0);
  std::vector<double> Eg(G);
  for (int g = 0; g < G; ++g) {
    Eg[g] = std::exp(o.lnEmin + g * o.dlnE);
    find_cs0_host(t, Eg[g] / 1000, o.sig_el[g], o.sig_ion[g], o.sig_exc[g], 0u);
    if (!std::isfinite(o.sig_el[g]) || !std::isfinite(o.sig_ion[g]) || !std::isfinite(o.sig_exc[g])) {
      err = "non-finite cross-section on the energy grid";
      return GASATT_E_TABLES;
    }
  }
  const double h = GASATT_PI / 180;
  const int ne = el.ne;
  for (int g = 0; g < G; ++g) {
    double le = std::log(Eg[g] / 1000);
    if (le < el.xInterp[0]) le = el.xInterp[0];
    if (le > el.xInterp[ne - 1]) le = el.xInterp[ne - 1];
    int i = 0;
    while (i < ne - 2 && le > el.xInterp[i + 1]) i++;
    const double a0 = (el.xInterp[i + 1] - le) / (el.xInterp[i + 1] - el.xInterp[i]);
    const double b0 = (le - el.xInterp[i]) / (el.xInterp[i + 1] - el.xInterp[i]);
    double *C = &o.cdf[(size_t)g * 181];
    double prev = 0;
    C[0] = 0;
    for (int k = 0; k <= 180; ++k) {
      const double vI = a0 * el.V[(size_t)i * 181 + k] + b0 * el.V[(size_t)(i + 1) * 181 + k];
      const double pdf = 2 * GASATT_PI * std::sin(k * h) * std::exp(vI) * 2;
      if (k > 0) C[k] = C[k - 1] + (prev + pdf) / 2 * h;
      prev = pdf;
    }
    const double tot = C[180];
    for (int k = 0; k <= 180; ++k) C[k] = C[k] / tot;
  }
  double vmax = 0;
  for (int g = 0; g <= G; ++g) {
    double sg, vg;
    if (g == G) {
      sg = o.sig_el[G - 1] + o.sig_ion[G - 1] + o.sig_exc[G - 1];
      vg = c;
    } else {
      const double s0 = o.sig_el[g] + o.sig_ion[g] + o.sig_exc[g];
      const double s1 = (g + 1 < G) ? o.sig_el[g + 1] + o.sig_ion[g + 1] + o.sig_exc[g + 1] : s0;
      sg = s0 > s1 ? s0 : s1;
      const double Eu = (g + 1 < G) ? Eg[g + 1] : Eg[g];
      const double eps = Eu * qe / (me * c * c);
      vg = c * std::sqrt(eps * (2 + eps)) / (1 + eps);
    }
    if (sg * vg > vmax) vmax = sg * vg;
  }
  o.sigv_max = vmax;
  o.nu_max = n_gas * vmax;
  // mean excitation energy loss sum_j k_j s_j / sum_j s_j over the terms above
  // threshold (electron_transport.cu:207-219, get_ImpExc2.m; q0 cancels)
  o.exc_kmin = 1e300;
  for (int i = 0; i < t->n_exc; ++i) o.exc_kmin = std::min(o.exc_kmin, t->t_exc[i]);
  for (int g = 0; g < G; ++g) {
    const double T = Eg[g];
    double k1 = 0, k2 = 0;
    for (int i = 0; i < t->n_exc; ++i) {
      const double k = t->t_exc[i], A = t->t_exc[t->n_exc + i], om = t->t_exc[2 * t->n_exc + i];
      const double nu = t->t_exc[3 * t->n_exc + i], ga = t->t_exc[4 * t->n_exc + i];
      if (!(T > k)) continue;
      const double a = A / (k * k);
      const double b = std::pow(k / T, om);
      const double cc = std::pow(1 - std::pow(k / T, ga), nu);
      k1 = k1 + a * b * cc * k;
      k2 = k2 + a * b * cc;
    }
    o.edep[g] = k2 > 0 ? k1 / k2 : 0.0;
  }
  o.n_exc = t->n_exc;
  for (int j = 0; j < 5; ++j)
    for (int i = 0; i < t->n_exc; ++i) o.exc[j][i] = t->t_exc[j * t->n_exc + i];
  return GASATT_OK;
}

}  // namespace gasatt
