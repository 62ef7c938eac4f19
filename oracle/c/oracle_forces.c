/*
 * FP64 C/OpenMP restatement of prolix's implicit-solvent energy and forces.
 *
 * TEST INFRASTRUCTURE ONLY: used by the tests as a fast checker at sizes the
 * NumPy oracle (oracle/gbsa.py, oracle/bonded.py) cannot reach quickly, and
 * by bench.py as the CPU baseline.  Same formulas and the same reference
 * citations as the NumPy oracle:
 *   pair integral, Born radii, GB, ACE  prolix physics/generalized_born.py:32-263, 600-648
 *   Coulomb, LJ with exclusion scales   physics/optimization.py:21-297
 *   chain rule through the Born radii   physics/analytical_forces.py:167-292
 *   bond, angle, periodic torsion       physics/bonded.py:20-141
 * Unique pairs are visited once per pass (i < j) with per-thread force
 * buffers reduced at the end.  cutoff <= 0 means all pairs; gb_cutoff < 0
 * means "same as cutoff"; a GB cutoff > 0 applies the neighbour-list clamps
 * of generalized_born.py:300-337.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SAFE_EPS 1e-12

static double pair_integral(double r, double rho, double s) {
  if (!(r + s > rho)) return 0.0;
  double d = fabs(r - s);
  double L = fmax(fmax(rho, d), 1e-4), U = fmax(r + s, 1e-4), rs = fmax(r, 1e-4);
  double il = 1.0 / L, iu = 1.0 / U;
  return 0.5 * (il - iu) + 0.25 * log(L / U) / rs + 0.125 * (r - s * s / rs) * (iu * iu - il * il);
}

static double pair_integral_dr(double r, double rho, double s) {
  if (!(r + s > rho)) return 0.0;
  double d = fabs(r - s);
  int use_d = d > rho;
  double Lraw = use_d ? d : rho;
  double L = fmax(Lraw, 1e-4);
  double dL = (use_d && Lraw > 1e-4) ? ((r - s) > 0 ? 1.0 : ((r - s) < 0 ? -1.0 : 0.0)) : 0.0;
  double Uraw = r + s, U = fmax(Uraw, 1e-4), dU = Uraw > 1e-4 ? 1.0 : 0.0;
  double rs = fmax(r, 1e-4), drs = r > 1e-4 ? 1.0 : 0.0;
  double il = 1.0 / L, iu = 1.0 / U, lg = log(L / U);
  double t1 = 0.5 * (-dL * il * il + dU * iu * iu);
  double t2 = 0.25 * ((dL / L - dU / U) / rs - lg * drs / (rs * rs));
  double a = r - s * s / rs, da = 1.0 + s * s * drs / (rs * rs);
  double b = iu * iu - il * il, db = -2.0 * dU * iu * iu * iu + 2.0 * dL * il * il * il;
  return t1 + t2 + 0.125 * (da * b + a * db);
}

typedef struct {
  int n;
  const double *pos, *q, *sigma, *eps, *radii, *sr;
  int n_excl;
  const int *excl;       /* (n_excl, 2) i < j */
  const int *excl_kind;  /* 0 excluded, 1 1-4 */
  double lj14, coul14, eps_in, eps_out, k_gb, k_coul, cutoff, gb_cutoff;
  int n_bond;
  const int *bond;
  const double *bond_par;
  int n_angle;
  const int *angle;
  const double *angle_par;
  int n_tors, n_terms;
  const int *tors;
  const double *tors_par;
} pb2o_system;

/* energies[9]: bond angle dihedral cmap(0) lj coulomb gb nonpolar total; forces (n, 3) */
int pb2o_energy_forces(const pb2o_system *S, double *energies, double *forces, int n_threads) {
  const int n = S->n;
  const double *x = S->pos;
  const double gbc = S->gb_cutoff < 0 ? S->cutoff : S->gb_cutoff;
  const int clamp = gbc > 0;
  const double gc2 = gbc > 0 ? gbc * gbc : 0.0, cc2 = S->cutoff > 0 ? S->cutoff * S->cutoff : 0.0;
  const double pref = -0.5 * S->k_gb * (1.0 / S->eps_in - 1.0 / S->eps_out);
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
  const int nt = omp_get_max_threads();
#else
  const int nt = 1;
#endif
  double *ro = malloc(sizeof(double) * n), *rad = malloc(sizeof(double) * n);
  double *isum = calloc((size_t)n * nt, sizeof(double));
  double *born = malloc(sizeof(double) * n), *dbdi = malloc(sizeof(double) * n);
  double *dedb = calloc((size_t)n * nt, sizeof(double));
  double *f = calloc((size_t)n * 3 * nt, sizeof(double));
  double *scv = malloc(sizeof(double) * (size_t)n * nt), *sce = malloc(sizeof(double) * (size_t)n * nt);
  int *eoff = calloc(n + 1, sizeof(int)), *elist = malloc(sizeof(int) * (size_t)(S->n_excl + 1));
  double *ev = malloc(sizeof(double) * (size_t)(S->n_excl + 1)), *ee = malloc(sizeof(double) * (size_t)(S->n_excl + 1));
  if (!ro || !rad || !isum || !born || !dbdi || !dedb || !f || !scv || !sce || !eoff || !elist || !ev || !ee)
    return -1;
  for (int i = 0; i < n; ++i) {
    rad[i] = clamp ? fmax(S->radii[i], 1e-6) : S->radii[i];
    ro[i] = rad[i] - 0.09;
    if (clamp) ro[i] = fmax(ro[i], 1e-4);
  }
  /* exclusions by lower atom (CSR) */
  for (int k = 0; k < S->n_excl; ++k) eoff[S->excl[2 * k] + 1]++;
  for (int i = 0; i < n; ++i) eoff[i + 1] += eoff[i];
  {
    int *cur = calloc(n, sizeof(int));
    for (int k = 0; k < S->n_excl; ++k) {
      int i = S->excl[2 * k], slot = eoff[i] + cur[i]++;
      elist[slot] = S->excl[2 * k + 1];
      ev[slot] = S->excl_kind[k] ? S->lj14 : 0.0;
      ee[slot] = S->excl_kind[k] ? S->coul14 : 0.0;
    }
    free(cur);
  }
  double e_lj = 0, e_coul = 0, e_gb = 0, e_ace = 0;
  /* pass 1: descreening sums */
#pragma omp parallel
  {
#ifdef _OPENMP
    const int t = omp_get_thread_num();
#else
    const int t = 0;
#endif
    double *my = isum + (size_t)t * n;
#pragma omp for schedule(dynamic, 16)
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) {
        double dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1], dz = x[3 * i + 2] - x[3 * j + 2];
        double r2 = dx * dx + dy * dy + dz * dz;
        double r = sqrt(r2 + SAFE_EPS);
        if (gc2 > 0 && r >= gbc) continue;
        my[i] += pair_integral(r, ro[i], S->sr[j]);
        my[j] += pair_integral(r, ro[j], S->sr[i]);
      }
  }
  for (int i = 0; i < n; ++i) {
    double I = 0;
    for (int t = 0; t < nt; ++t) I += isum[(size_t)t * n + i];
    double psi = ro[i] * I;
    double th = tanh(psi - 0.8 * psi * psi + 4.85 * psi * psi * psi);
    double dr = clamp ? fmax(rad[i], 1e-4) : rad[i];
    double ib = 1.0 / ro[i] - th / dr;
    int clamped = 0;
    if (clamp && ib < 1e-4) { ib = 1e-4; clamped = 1; }
    born[i] = 1.0 / ib;
    dbdi[i] = clamped ? 0.0 : born[i] * born[i] * (1.0 - th * th) / dr * (1.0 - 1.6 * psi + 14.55 * psi * psi) * ro[i];
    double q = S->q[i];
    double rnm = (S->radii[i] - 0.09) / 10.0 + 0.009;
    double xr = rnm / (born[i] / 10.0);
    double ace = 28.3919551 * (rnm + 0.14) * (rnm + 0.14) * pow(xr, 6) * 0.239006;
    e_gb += pref * q * q / born[i];
    e_ace += ace;
    dedb[i] = -pref * q * q / (born[i] * born[i]) - 6.0 * ace / born[i];
  }
  /* pass 2: GB pairs, Coulomb, LJ */
#pragma omp parallel reduction(+ : e_lj, e_coul, e_gb)
  {
#ifdef _OPENMP
    const int t = omp_get_thread_num();
#else
    const int t = 0;
#endif
    double *myf = f + (size_t)t * 3 * n, *myd = dedb + (size_t)t * n;
    double *sv = scv + (size_t)t * n, *se = sce + (size_t)t * n;
    for (int j = 0; j < n; ++j) sv[j] = se[j] = 1.0;
#pragma omp for schedule(dynamic, 16)
    for (int i = 0; i < n; ++i) {
      for (int k = eoff[i]; k < eoff[i + 1]; ++k) { sv[elist[k]] = ev[k]; se[elist[k]] = ee[k]; }
      for (int j = i + 1; j < n; ++j) {
        double dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1], dz = x[3 * i + 2] - x[3 * j + 2];
        double r2 = dx * dx + dy * dy + dz * dz;
        double g = 0.0, qq = S->q[i] * S->q[j];
        double rg2 = r2 + SAFE_EPS;
        if (!(gc2 > 0 && sqrt(rg2) >= gbc)) {
          double D = born[i] * born[j], ex = exp(-rg2 / (4.0 * D));
          double f2 = rg2 + D * ex, fv = sqrt(f2), if3 = 1.0 / (f2 * fv);
          e_gb += 2.0 * pref * qq / fv;
          g += 2.0 * pref * qq * (1.0 - 0.25 * ex) * if3;
          double c = -pref * qq * ex * (1.0 + rg2 / (4.0 * D)) * if3;
          myd[i] += c * born[j];
          myd[j] += c * born[i];
        }
        if (r2 > 0 && !(cc2 > 0 && r2 >= cc2)) {
          double ir = 1.0 / sqrt(r2), ir2 = ir * ir;
          double ec = S->k_coul * qq * se[j] * ir;
          e_coul += ec;
          g += ec * ir2;
          double sig = 0.5 * (fmax(S->sigma[i], 1e-6) + fmax(S->sigma[j], 1e-6));
          double ep = sqrt(S->eps[i] * S->eps[j]) * sv[j];
          double s2 = sig * sig * ir2, s6 = s2 * s2 * s2;
          e_lj += 4.0 * ep * (s6 * s6 - s6);
          g += 4.0 * ep * (12.0 * s6 * s6 - 6.0 * s6) * ir2;
        }
        myf[3 * i] += g * dx; myf[3 * i + 1] += g * dy; myf[3 * i + 2] += g * dz;
        myf[3 * j] -= g * dx; myf[3 * j + 1] -= g * dy; myf[3 * j + 2] -= g * dz;
      }
      for (int k = eoff[i]; k < eoff[i + 1]; ++k) { sv[elist[k]] = 1.0; se[elist[k]] = 1.0; }
    }
  }
  /* reduce dE/dB, then pass 3: chain rule */
  for (int t = 1; t < nt; ++t)
    for (int i = 0; i < n; ++i) dedb[i] += dedb[(size_t)t * n + i];
  double *dedi = dbdi; /* reuse: dE/dI = dE/dB dB/dI */
  for (int i = 0; i < n; ++i) dedi[i] = dedb[i] * dbdi[i];
#pragma omp parallel
  {
#ifdef _OPENMP
    const int t = omp_get_thread_num();
#else
    const int t = 0;
#endif
    double *myf = f + (size_t)t * 3 * n;
#pragma omp for schedule(dynamic, 16)
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) {
        double dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1], dz = x[3 * i + 2] - x[3 * j + 2];
        double r = sqrt(dx * dx + dy * dy + dz * dz + SAFE_EPS);
        if (gc2 > 0 && r >= gbc) continue;
        double g = (dedi[i] * pair_integral_dr(r, ro[i], S->sr[j]) +
                    dedi[j] * pair_integral_dr(r, ro[j], S->sr[i])) / r;
        myf[3 * i] -= g * dx; myf[3 * i + 1] -= g * dy; myf[3 * i + 2] -= g * dz;
        myf[3 * j] += g * dx; myf[3 * j + 1] += g * dy; myf[3 * j + 2] += g * dz;
      }
  }
  for (int i = 0; i < 3 * n; ++i) {
    double v = 0;
    for (int t = 0; t < nt; ++t) v += f[(size_t)t * 3 * n + i];
    forces[i] = v;
  }
  /* bonded */
  double e_b = 0, e_a = 0, e_d = 0;
  for (int k = 0; k < S->n_bond; ++k) {
    int i = S->bond[2 * k], j = S->bond[2 * k + 1];
    double d[3], r = 0;
    for (int c = 0; c < 3; ++c) { d[c] = x[3 * i + c] - x[3 * j + c]; r += d[c] * d[c]; }
    r = sqrt(r);
    double r0 = S->bond_par[2 * k], kk = S->bond_par[2 * k + 1];
    e_b += 0.5 * kk * (r - r0) * (r - r0);
    for (int c = 0; c < 3; ++c) { double g = kk * (r - r0) / r * d[c]; forces[3 * i + c] -= g; forces[3 * j + c] += g; }
  }
  for (int k = 0; k < S->n_angle; ++k) {
    int i = S->angle[3 * k], j = S->angle[3 * k + 1], l = S->angle[3 * k + 2];
    double a[3], b[3], la = 0, lb = 0, dt = 0;
    for (int c = 0; c < 3; ++c) { a[c] = x[3 * i + c] - x[3 * j + c]; b[c] = x[3 * l + c] - x[3 * j + c]; }
    for (int c = 0; c < 3; ++c) { la += a[c] * a[c]; lb += b[c] * b[c]; dt += a[c] * b[c]; }
    la = sqrt(la); lb = sqrt(lb);
    double den = la * lb + 1e-8, cs = dt / den;
    int clipped = cs < -0.999999 || cs > 0.999999;
    cs = fmin(fmax(cs, -0.999999), 0.999999);
    double th = acos(cs), th0 = S->angle_par[2 * k], kk = S->angle_par[2 * k + 1];
    e_a += 0.5 * kk * (th - th0) * (th - th0);
    double s = kk * (th - th0) * (clipped ? 0.0 : -1.0 / sqrt(1.0 - cs * cs));
    for (int c = 0; c < 3; ++c) {
      double gi = s * (b[c] / den - dt * lb / (den * den * la) * a[c]);
      double gk = s * (a[c] / den - dt * la / (den * den * lb) * b[c]);
      forces[3 * i + c] -= gi; forces[3 * j + c] += gi + gk; forces[3 * l + c] -= gk;
    }
  }
  for (int k = 0; k < S->n_tors; ++k) {
    const int *id = S->tors + 4 * k;
    double ri[3], rj[3], rk[3], rl[3];
    for (int c = 0; c < 3; ++c) { ri[c] = x[3 * id[0] + c]; rj[c] = x[3 * id[1] + c]; rk[c] = x[3 * id[2] + c]; rl[c] = x[3 * id[3] + c]; }
    double b0[3], b1[3], b2[3];
    for (int c = 0; c < 3; ++c) { b0[c] = ri[c] - rj[c]; b1[c] = rk[c] - rj[c]; b2[c] = rl[c] - rk[c]; }
    double nb1 = sqrt(b1[0] * b1[0] + b1[1] * b1[1] + b1[2] * b1[2]) + 1e-8, u[3];
    for (int c = 0; c < 3; ++c) u[c] = b1[c] / nb1;
    double p0 = b0[0] * u[0] + b0[1] * u[1] + b0[2] * u[2], p2 = b2[0] * u[0] + b2[1] * u[1] + b2[2] * u[2];
    double v[3], w[3];
    for (int c = 0; c < 3; ++c) { v[c] = b0[c] - p0 * u[c]; w[c] = b2[c] - p2 * u[c]; }
    double uv[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
    double phi = atan2(uv[0] * w[0] + uv[1] * w[1] + uv[2] * w[2], v[0] * w[0] + v[1] * w[1] + v[2] * w[2]);
    double F[3], G[3], H[3];
    for (int c = 0; c < 3; ++c) { F[c] = ri[c] - rj[c]; G[c] = rj[c] - rk[c]; H[c] = rl[c] - rk[c]; }
    double A[3] = {F[1] * G[2] - F[2] * G[1], F[2] * G[0] - F[0] * G[2], F[0] * G[1] - F[1] * G[0]};
    double B[3] = {H[1] * G[2] - H[2] * G[1], H[2] * G[0] - H[0] * G[2], H[0] * G[1] - H[1] * G[0]};
    double lg = sqrt(G[0] * G[0] + G[1] * G[1] + G[2] * G[2]);
    double a2 = A[0] * A[0] + A[1] * A[1] + A[2] * A[2], b2n = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
    double fg = F[0] * G[0] + F[1] * G[1] + F[2] * G[2], hg = H[0] * G[0] + H[1] * G[1] + H[2] * G[2];
    double dedphi = 0;
    for (int t = 0; t < S->n_terms; ++t) {
      const double *p = S->tors_par + ((size_t)k * S->n_terms + t) * 3;
      double ang = p[0] * phi - p[1];
      e_d += p[2] * (1.0 + cos(ang));
      dedphi += -p[2] * p[0] * sin(ang);
    }
    for (int c = 0; c < 3; ++c) {
      double gi = -lg / a2 * A[c], gl = lg / b2n * B[c];
      double ta = fg / (a2 * lg) * A[c], tb = hg / (b2n * lg) * B[c];
      double gj = -gi + ta - tb, gk = -gl - ta + tb;
      forces[3 * id[0] + c] -= dedphi * gi; forces[3 * id[1] + c] -= dedphi * gj;
      forces[3 * id[2] + c] -= dedphi * gk; forces[3 * id[3] + c] -= dedphi * gl;
    }
  }
  energies[0] = e_b; energies[1] = e_a; energies[2] = e_d; energies[3] = 0.0;
  energies[4] = e_lj; energies[5] = e_coul; energies[6] = e_gb; energies[7] = e_ace;
  energies[8] = e_b + e_a + e_d + e_lj + e_coul + e_gb + e_ace;
  free(ro); free(rad); free(isum); free(born); free(dbdi); free(dedb); free(f); free(scv); free(sce);
  free(eoff); free(elist); free(ev); free(ee);
  return 0;
}
