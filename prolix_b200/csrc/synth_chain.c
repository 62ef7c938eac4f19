/*
 * Host-side chain growth for the seeded synthetic systems.
 *
 * The random draws (bond lengths, bond angles and a set of candidate
 * dihedrals per atom) are made by the caller with NumPy's default_rng; this
 * file only does the geometry and the deterministic candidate selection, so
 * a given seed always produces the same coordinates.
 *
 * Placement rule for atom i (i >= 3): each candidate dihedral gives one
 * position through the natural-extension-reference-frame construction from
 * atoms i-3, i-2, i-1.  A candidate is feasible when every atom j <= i-3 is
 * at least `min_dist` away.  In extended mode the first feasible candidate
 * is taken; in compact mode the first feasible candidate inside the sphere
 * of radius `confine` is taken, else the feasible candidate closest to the
 * origin, which packs the chain into a globule.  When no candidate is
 * feasible, the one with the largest nearest-atom distance is taken.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define HASH_BITS 20
#define HASH_SIZE (1u << HASH_BITS)

typedef struct {
  int *head;  /* HASH_SIZE bucket heads */
  int *next;  /* per-atom chain */
  double cell;
} grid_t;

static unsigned cell_hash(long ix, long iy, long iz) {
  unsigned long long h = (unsigned long long)(ix * 73856093LL) ^
                         (unsigned long long)(iy * 19349663LL) ^
                         (unsigned long long)(iz * 83492791LL);
  h ^= h >> 29;
  h *= 0xbf58476d1ce4e5b9ULL;
  h ^= h >> 32;
  return (unsigned)(h & (HASH_SIZE - 1));
}

static void grid_insert(grid_t *g, const double *pos, int i) {
  long ix = (long)floor(pos[3 * i] / g->cell);
  long iy = (long)floor(pos[3 * i + 1] / g->cell);
  long iz = (long)floor(pos[3 * i + 2] / g->cell);
  unsigned h = cell_hash(ix, iy, iz);
  g->next[i] = g->head[h];
  g->head[h] = i;
}

/* Smallest distance from point p to any placed atom with index <= last. */
static double nearest(const grid_t *g, const double *pos, const double *p, int last,
                      double search) {
  double best2 = search * search;
  long cx = (long)floor(p[0] / g->cell);
  long cy = (long)floor(p[1] / g->cell);
  long cz = (long)floor(p[2] / g->cell);
  long r = (long)ceil(search / g->cell);
  for (long dx = -r; dx <= r; ++dx)
    for (long dy = -r; dy <= r; ++dy)
      for (long dz = -r; dz <= r; ++dz) {
        unsigned h = cell_hash(cx + dx, cy + dy, cz + dz);
        for (int j = g->head[h]; j >= 0; j = g->next[j]) {
          if (j > last) continue;
          double ex = pos[3 * j] - p[0], ey = pos[3 * j + 1] - p[1],
                 ez = pos[3 * j + 2] - p[2];
          double d2 = ex * ex + ey * ey + ez * ez;
          if (d2 < best2) best2 = d2;
        }
      }
  return sqrt(best2);
}

static void place(const double *a, const double *b, const double *c, double len,
                  double theta, double phi, double *out) {
  /* bc = unit(c - b); n = unit((b - a) x bc); m = n x bc */
  double bc[3] = {c[0] - b[0], c[1] - b[1], c[2] - b[2]};
  double nb = sqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]);
  for (int k = 0; k < 3; ++k) bc[k] /= nb;
  double ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double n[3] = {ab[1] * bc[2] - ab[2] * bc[1], ab[2] * bc[0] - ab[0] * bc[2],
                 ab[0] * bc[1] - ab[1] * bc[0]};
  double nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  if (nn < 1e-12) { /* collinear: pick any perpendicular */
    n[0] = -bc[1]; n[1] = bc[0]; n[2] = 0.0;
    nn = sqrt(n[0] * n[0] + n[1] * n[1]);
    if (nn < 1e-12) { n[0] = 0.0; n[1] = -bc[2]; n[2] = bc[1]; nn = sqrt(n[1] * n[1] + n[2] * n[2]); }
  }
  for (int k = 0; k < 3; ++k) n[k] /= nn;
  double m[3] = {n[1] * bc[2] - n[2] * bc[1], n[2] * bc[0] - n[0] * bc[2],
                 n[0] * bc[1] - n[1] * bc[0]};
  double d2x = -len * cos(theta);
  double d2y = len * sin(theta) * cos(phi);
  double d2z = len * sin(theta) * sin(phi);
  for (int k = 0; k < 3; ++k) out[k] = c[k] + d2x * bc[k] + d2y * m[k] + d2z * n[k];
}

static void grid_pop(grid_t *g, const double *pos, int i) {
  /* atoms leave in reverse insertion order, so i heads its bucket */
  long ix = (long)floor(pos[3 * i] / g->cell);
  long iy = (long)floor(pos[3 * i + 1] / g->cell);
  long iz = (long)floor(pos[3 * i + 2] / g->cell);
  unsigned h = cell_hash(ix, iy, iz);
  if (g->head[h] == i) g->head[h] = g->next[i];
}

static unsigned long long splitmix64(unsigned long long *s) {
  unsigned long long z = (*s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

/*
 * n atoms; lengths[i] is the bond (i-1, i); angles[i] the angle (i-2, i-1, i)
 * in radians; cand[i * ncand + k] the k-th candidate dihedral of atom i.
 * When no candidate of atom i is feasible the last few atoms are removed and
 * regrown with dihedrals from a splitmix64 stream seeded by `retry_seed`
 * (bounded: at most 64 * n regrowths in total).  chosen[i] receives the
 * dihedral used (NaN for i < 3).  Returns the number of atoms finally placed
 * without a feasible candidate, or -1 if memory ran out.
 */
int pb2_synth_grow_chain(int n, int ncand, const double *lengths, const double *angles,
                         const double *cand, int compact, double confine, double min_dist,
                         unsigned long long retry_seed, double *pos, double *chosen) {
  if (n <= 0) return 0;
  grid_t g;
  g.cell = min_dist > 0.5 ? min_dist : 0.5;
  g.head = (int *)malloc(sizeof(int) * HASH_SIZE);
  g.next = (int *)malloc(sizeof(int) * (size_t)n);
  unsigned char *regrow = (unsigned char *)calloc((size_t)n, 1);
  int *tries = (int *)calloc((size_t)n, sizeof(int));
  if (!g.head || !g.next || !regrow || !tries) {
    free(g.head); free(g.next); free(regrow); free(tries);
    return -1;
  }
  memset(g.head, 0xff, sizeof(int) * HASH_SIZE);
  unsigned long long rs = retry_seed;
  long long budget = 64LL * n;
  int infeasible = 0, inserted = 0;
  for (int i = 0; i < n; ++i) chosen[i] = NAN;
  pos[0] = pos[1] = pos[2] = 0.0;
  if (n > 1) { pos[3] = lengths[1]; pos[4] = 0.0; pos[5] = 0.0; }
  if (n > 2) {
    double th = angles[2];
    pos[6] = pos[3] - lengths[2] * cos(th);
    pos[7] = lengths[2] * sin(th);
    pos[8] = 0.0;
  }
  int i = 3;
  while (i < n) {
    while (inserted <= i - 3) grid_insert(&g, pos, inserted++);
    const double *a = pos + 3 * (i - 3), *b = pos + 3 * (i - 2), *c = pos + 3 * (i - 1);
    double best_score = 0.0, best_near = -1.0, p[3], keep[3] = {0, 0, 0}, keep_phi = NAN;
    int have_feasible = 0;
    for (int k = 0; k < ncand; ++k) {
      double phi = regrow[i] ? (double)(splitmix64(&rs) >> 11) * (2.0 * M_PI / 9007199254740992.0) - M_PI
                             : cand[(size_t)i * ncand + k];
      place(a, b, c, lengths[i], angles[i], phi, p);
      double d = nearest(&g, pos, p, i - 3, min_dist);
      if (d >= min_dist) {
        double r2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        int inside = !compact || r2 <= confine * confine;
        double score = inside ? 1.0 : -r2;
        if (!have_feasible || score > best_score) {
          have_feasible = 1;
          best_score = score;
          keep[0] = p[0]; keep[1] = p[1]; keep[2] = p[2];
          keep_phi = phi;
          if (inside) break;
        }
      } else if (!have_feasible && d > best_near) {
        best_near = d;
        keep[0] = p[0]; keep[1] = p[1]; keep[2] = p[2];
        keep_phi = phi;
      }
    }
    if (!have_feasible && budget > 0 && i > 6) {
      /* back up a few atoms (more on repeated failure) and regrow them */
      budget -= 1;
      int back = 2 + (tries[i] < 6 ? tries[i] : 6);
      tries[i] += 1;
      int to = i - back;
      if (to < 4) to = 4;
      for (int k = to; k <= i; ++k) regrow[k] = 1;
      while (inserted > to - 3) grid_pop(&g, pos, --inserted);
      i = to;
      continue;
    }
    if (!have_feasible) ++infeasible;
    pos[3 * i] = keep[0]; pos[3 * i + 1] = keep[1]; pos[3 * i + 2] = keep[2];
    chosen[i] = keep_phi;
    ++i;
  }
  free(g.head);
  free(g.next);
  free(regrow);
  free(tries);
  return infeasible;
}
