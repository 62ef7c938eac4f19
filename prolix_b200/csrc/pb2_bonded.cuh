// Bonded terms: harmonic bonds, Urey-Bradley springs and angles, periodic
// torsions, periodic and harmonic impropers, CMAP and the explicit 1-4
// exception pairs, one term per call of bonded_term.  Used by the bonded
// kernel (pb2_bonded.cu) and, as tail work after the tiles, by the chain-rule
// pair pass (pb2_pair.cu).  See pb2_bonded.cu for the formulas' references.
#pragma once

#include "pb2_common.cuh"
#include "pb2_kernels.cuh"

namespace pb2 {


struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 ld3(const BondedArgs &a, int i) { return {a.x[i], a.y[i], a.z[i]}; }
__device__ __forceinline__ D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross(D3 a, D3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ D3 scale(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }

__device__ __forceinline__ void add_force(const BondedArgs &a, int i, D3 f) {
  atomic_add_fix(&a.fx[i], to_fix(f.x, kForceScale));
  atomic_add_fix(&a.fy[i], to_fix(f.y, kForceScale));
  atomic_add_fix(&a.fz[i], to_fix(f.z, kForceScale));
}

__device__ __forceinline__ void add_energy(const BondedArgs &a, int atom, int term, double e) {
  if (!a.energy_mode) return;
  const int s = a.atom_sys[atom];
  atomic_add_fix(&a.energy[(size_t)s * PB2_NTERMS + term], to_fix(e, kEnergyScale));
}

// Dihedral angle and its gradient w.r.t. the four atoms.
static __device__ void dihedral(const BondedArgs &a, int i, int j, int k, int l, double &phi, D3 g[4]) {
  const D3 ri = ld3(a, i), rj = ld3(a, j), rk = ld3(a, k), rl = ld3(a, l);
  const D3 b0 = sub(ri, rj), b1 = sub(rk, rj), b2 = sub(rl, rk);
  const double nb1 = sqrt(dot(b1, b1)) + 1e-8;
  const D3 u = scale(b1, 1.0 / nb1);
  const D3 v = sub(b0, scale(u, dot(b0, u)));
  const D3 w = sub(b2, scale(u, dot(b2, u)));
  phi = atan2(dot(cross(u, v), w), dot(v, w));
  const D3 F = sub(ri, rj), G = sub(rj, rk), H = sub(rl, rk);
  const D3 A = cross(F, G), B = cross(H, G);
  const double lg = sqrt(dot(G, G));
  const double a2 = dot(A, A), b2n = dot(B, B);
  const double fg = dot(F, G), hg = dot(H, G);
  g[0] = scale(A, -lg / a2);
  g[3] = scale(B, lg / b2n);
  const D3 ta = scale(A, fg / (a2 * lg)), tb = scale(B, hg / (b2n * lg));
  g[1] = {-g[0].x + ta.x - tb.x, -g[0].y + ta.y - tb.y, -g[0].z + ta.z - tb.z};
  g[2] = {-g[3].x - ta.x + tb.x, -g[3].y - ta.y + tb.y, -g[3].z - ta.z + tb.z};
}

// Total bonded terms of the batch (the index range of bonded_term).
__device__ __forceinline__ int bonded_total(const BondedArgs &a) {
  return a.n_bond + a.n_angle + a.n_tors + a.n_cmap + a.n_exc;
}

// Term t of the batch: bonds (then Urey-Bradley springs), angles, torsions
// and impropers, CMAP, exception pairs, in that index order.  Inlined into
// the bonded kernel; bonded_term_call keeps it out of line for the chain
// pass, whose hot loop should not grow.
static __device__ __forceinline__ void bonded_term(const BondedArgs &a, int t) {
  {
    int u = t;
    if (u < a.n_bond) {
      const int2 id = a.bond_idx[u];
      const double2 p = a.bond_par[u];
      const D3 d = sub(ld3(a, id.x), ld3(a, id.y));
      const double r = sqrt(dot(d, d));
      const double g = p.y * (r - p.x) / r;
      add_force(a, id.x, scale(d, -g));
      add_force(a, id.y, scale(d, g));
      add_energy(a, id.x, u < a.n_bond_plain ? PB2_TERM_BOND : PB2_TERM_UREY_BRADLEY,
                 0.5 * p.y * (r - p.x) * (r - p.x));
      return;
    }
    u -= a.n_bond;
    if (u < a.n_angle) {
      const int4 id = a.angle_idx[u];
      const double2 p = a.angle_par[u];
      const D3 rj = ld3(a, id.y);
      const D3 va = sub(ld3(a, id.x), rj), vb = sub(ld3(a, id.z), rj);
      const double la = sqrt(dot(va, va)), lb = sqrt(dot(vb, vb));
      const double den = la * lb + 1e-8;
      const double dt = dot(va, vb);
      double c = dt / den;
      const bool clipped = (c < -0.999999) || (c > 0.999999);
      c = fmin(fmax(c, -0.999999), 0.999999);
      const double th = acos(c);
      const double dedth = p.y * (th - p.x);
      const double dthdc = clipped ? 0.0 : -1.0 / sqrt(1.0 - c * c);
      const double s = dedth * dthdc;
      const double ca = dt * lb / (den * den * la), cb = dt * la / (den * den * lb);
      const D3 gi = {s * (vb.x / den - ca * va.x), s * (vb.y / den - ca * va.y), s * (vb.z / den - ca * va.z)};
      const D3 gk = {s * (va.x / den - cb * vb.x), s * (va.y / den - cb * vb.y), s * (va.z / den - cb * vb.z)};
      add_force(a, id.x, scale(gi, -1.0));
      add_force(a, id.y, {gi.x + gk.x, gi.y + gk.y, gi.z + gk.z});
      add_force(a, id.z, scale(gk, -1.0));
      add_energy(a, id.x, PB2_TERM_ANGLE, 0.5 * p.y * (th - p.x) * (th - p.x));
      return;
    }
    u -= a.n_angle;
    if (u < a.n_tors) {
      const int4 id = a.tors_idx[u];
      const double4 p = a.tors_par[u];
      double phi;
      D3 g[4];
      dihedral(a, id.x, id.y, id.z, id.w, phi, g);
      double e, dedphi;
      int term;
      if (p.w == kTorsHarmonic) {  // (k, phi0): k d^2, d wrapped into [-pi, pi)
        const double pi = 3.141592653589793, two_pi = 6.283185307179586;
        double d = phi - p.y + pi;
        d = d - two_pi * floor(d / two_pi) - pi;
        e = p.x * d * d;
        dedphi = 2.0 * p.x * d;
        term = PB2_TERM_IMPROPER;
      } else {  // (n, phase, k): k (1 + cos(n phi - phase))
        const double ang = p.x * phi - p.y;
        e = p.z * (1.0 + cos(ang));
        dedphi = -p.z * p.x * sin(ang);
        term = p.w == kTorsImproper ? PB2_TERM_IMPROPER : PB2_TERM_DIHEDRAL;
      }
      const int ids[4] = {id.x, id.y, id.z, id.w};
#pragma unroll
      for (int c = 0; c < 4; ++c) add_force(a, ids[c], scale(g[c], -dedphi));
      add_energy(a, id.x, term, e);
      return;
    }
    u -= a.n_tors;
    if (u < a.n_cmap) {
      const int32_t *row = a.cmap_idx + (size_t)u * 6;
      const int m = row[5];
      const int G = a.cmap_grid[m];
      const double *coef = a.cmap_coeff + a.cmap_map_off[m];
      double phi, psi;
      D3 gphi[4], gpsi[4];
      dihedral(a, row[0], row[1], row[2], row[3], phi, gphi);
      dihedral(a, row[1], row[2], row[3], row[4], psi, gpsi);
      const double two_pi = 6.283185307179586;
      const double delta = two_pi / G;
      const double pn = fmod(phi + two_pi, two_pi);
      const double sn = fmod(psi + two_pi, two_pi);
      if (!(isfinite(pn) && isfinite(sn))) return;  // non-finite state: flagged by the integrator
      int ia = (int)floor(pn / delta);
      int ib = (int)floor(sn / delta);
      ia = min(max(ia % G, 0), G - 1);
      ib = min(max(ib % G, 0), G - 1);
      const double da = pn / delta - ia, db = sn / delta - ib;
      const double *c = coef + ((size_t)ia * G + ib) * 16;
      double e = 0.0, ea = 0.0, eb = 0.0;
      const double pa[4] = {1.0, da, da * da, da * da * da};
      const double pb[4] = {1.0, db, db * db, db * db * db};
      const double dpa[4] = {0.0, 1.0, 2.0 * da, 3.0 * da * da};
      const double dpb[4] = {0.0, 1.0, 2.0 * db, 3.0 * db * db};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const double cij = c[i * 4 + j];
          e += cij * pa[i] * pb[j];
          ea += cij * dpa[i] * pb[j];
          eb += cij * pa[i] * dpb[j];
        }
      ea /= delta;
      eb /= delta;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        add_force(a, row[k], scale(gphi[k], -ea));
        add_force(a, row[k + 1], scale(gpsi[k], -eb));
      }
      add_energy(a, row[0], PB2_TERM_CMAP, e);
      return;
    }
    u -= a.n_cmap;
    {  // explicit 1-4 exception pair (bonded.py:211-228)
      const int2 id = a.exc_idx[u];
      const double4 p = a.exc_par[u];
      const D3 d = sub(ld3(a, id.x), ld3(a, id.y));
      const double r = sqrt(dot(d, d) + 1e-12);
      const double inv = 1.0 / r;
      double e = 0.0, dedr = 0.0;
      if (a.terms & PB2_USE_LJ) {
        const double sr = p.y * inv, s2 = sr * sr, s6 = s2 * s2 * s2;
        e += 4.0 * p.z * (s6 * s6 - s6);
        dedr += 4.0 * p.z * (6.0 * s6 - 12.0 * s6 * s6) * inv;
      }
      if (a.terms & PB2_USE_COULOMB) {
        const double ec = p.x * inv;
        e += ec;
        dedr -= ec * inv;
      }
      const double g = dedr * inv;
      add_force(a, id.x, scale(d, -g));
      add_force(a, id.y, scale(d, g));
      add_energy(a, id.x, PB2_TERM_EXCEPTION, e);
    }
  }
}

static __device__ __noinline__ void bonded_term_call(const BondedArgs &a, int t) { bonded_term(a, t); }

}  // namespace pb2
