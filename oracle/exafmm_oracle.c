/* CPU restatement of the exafmm-beta Laplace FMM path (spherical-harmonic
 * expansions, adaptive octree, dual tree traversal).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the GPU engine is checked
 * against; the product library never links it and never falls back to it.
 * It is pinned to the reference itself (the reference headers compiled in
 * place as oracle/_ref/libexafmm_ref.so) by tests/test_oracle.py.
 *
 * All citations are paths inside the exafmm-beta source tree.
 */
#define _GNU_SOURCE
#include "exafmm_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

/* ------------------------------------------------------------------------ */
/* Expansion tables (kernels/laplace.h:116-148).                             */
/* The reference scales Anm by 1/EPS and Cnm, M2M, L2L by EPS; the factors   */
/* cancel exactly in real arithmetic, so they are left out here.             */
/* ------------------------------------------------------------------------ */
typedef struct {
  int P;
  double *pref;  /* sqrt((n-|m|)!/(n+|m|)!), n < 2P, index n*n+n+m */
  double *anm;   /* (-1)^n / sqrt((n-m)!(n+m)!), n < 2P             */
  double *cjk;   /* M2L coefficient, real: i^(|k-m|-|k|-|m|) (-1)^j A_n^m A_j^k / A_{j+n}^{m-k} */
} tables_t;

#define ORACLE_PMAX 40
static tables_t *g_tables[ORACLE_PMAX + 1];

static double factorial(int k) {
  double f = 1.0;
  for (int i = 2; i <= k; i++) f *= i;
  return f;
}

static int sgn_pow(int e) { return (e & 1) ? -1 : 1; }

static const tables_t *tables_for(int P) {
  if (P < 1 || P > ORACLE_PMAX) return NULL;
  if (g_tables[P]) return g_tables[P];
  tables_t *t = (tables_t *)calloc(1, sizeof(tables_t));
  t->P = P;
  int Q = 2 * P;
  t->pref = (double *)malloc(sizeof(double) * Q * Q);
  t->anm = (double *)malloc(sizeof(double) * Q * Q);
  for (int n = 0; n < Q; n++) {
    for (int m = -n; m <= n; m++) {
      int am = abs(m);
      t->pref[n * n + n + m] = sqrt(factorial(n - am) / factorial(n + am));
      t->anm[n * n + n + m] = sgn_pow(n) / sqrt(factorial(n - m) * factorial(n + m));
    }
  }
  t->cjk = (double *)malloc(sizeof(double) * P * P * P * P);
  for (int j = 0, jk = 0; j < P; j++) {
    for (int k = -j; k <= j; k++, jk++) {
      for (int n = 0, nm = 0; n < P; n++) {
        for (int m = -n; m <= n; m++, nm++) {
          int e = abs(k - m) - abs(k) - abs(m);          /* always even and <= 0 */
          int jnkm = (j + n) * (j + n) + j + n + m - k;
          t->cjk[jk * P * P + nm] = sgn_pow(e / 2) * sgn_pow(j) *
                                     t->anm[nm] * t->anm[jk] / t->anm[jnkm];
        }
      }
    }
  }
  g_tables[P] = t;
  return t;
}

/* cart2sph (kernels/laplace.h:29-33). */
static void to_sph(const double d[3], double *r, double *theta, double *phi) {
  *r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  *theta = (*r == 0.0) ? 0.0 : acos(d[2] / *r);
  *phi = atan2(d[1], d[0]);
}

/* Regular solid harmonics rho^n P_n^m(cos a) pref e^{imb} and their polar
 * derivative, 0 <= |m| <= n < P (kernels/laplace.h:48-80).  P_n^m carries the
 * Condon-Shortley phase; the -m slots hold the conjugates. */
static void regular(const tables_t *t, double rho, double a, double b, cplx *Y, cplx *Yt) {
  const int P = t->P;
  const double c = cos(a), s = sin(a);
  double pmm = 1.0, rhom = 1.0;
  for (int m = 0; m < P; m++) {
    const cplx e = cexp(I * (m * b));
    double pa = pmm;                         /* P_m^m     */
    double pb = c * (2 * m + 1) * pmm;       /* P_{m+1}^m */
    int i = m * m + 2 * m;
    Y[i] = rhom * pa * t->pref[i] * e;
    Y[m * m] = conj(Y[i]);
    Yt[i] = rhom * (pb - (m + 1) * c * pa) / s * t->pref[i] * e;
    double rhon = rhom * rho;
    for (int n = m + 1; n < P; n++) {
      int ip = n * n + n + m, in = n * n + n - m;
      Y[ip] = rhon * pb * t->pref[ip] * e;
      Y[in] = conj(Y[ip]);
      double pc = (c * (2 * n + 1) * pb - (n + m) * pa) / (n - m + 1);  /* P_{n+1}^m */
      Yt[ip] = rhon * ((n - m + 1) * pc - (n + 1) * c * pb) / s * t->pref[ip] * e;
      pa = pb;
      pb = pc;
      rhon *= rho;
    }
    rhom *= rho;
    pmm = -pmm * (2 * m + 1) * s;
  }
}

/* Singular solid harmonics rho^{-n-1} P_n^m(cos a) pref e^{imb}, n < 2P
 * (kernels/laplace.h:83-113). */
static void singular(const tables_t *t, double rho, double a, double b, cplx *Y) {
  const int Q = 2 * t->P;
  const double c = cos(a), s = sin(a), inv = 1.0 / rho;
  double pmm = 1.0, rhom = inv;
  for (int m = 0; m < Q; m++) {
    const cplx e = cexp(I * (m * b));
    double pa = pmm, pb = c * (2 * m + 1) * pmm;
    int i = m * m + 2 * m;
    Y[i] = rhom * pmm * t->pref[i] * e;
    Y[m * m] = conj(Y[i]);
    double rhon = rhom * inv;
    for (int n = m + 1; n < Q; n++) {
      int ip = n * n + n + m, in = n * n + n - m;
      Y[ip] = rhon * pb * t->pref[ip] * e;
      Y[in] = conj(Y[ip]);
      double pc = (c * (2 * n + 1) * pb - (n + m) * pa) / (n - m + 1);
      pa = pb;
      pb = pc;
      rhon *= inv;
    }
    rhom *= inv;
    pmm = -pmm * (2 * m + 1) * s;
  }
}

/* Expansion coefficient (n, m) for any sign of m from the m >= 0 storage. */
static inline cplx coef(const cplx *E, int n, int m) {
  return m >= 0 ? E[n * (n + 1) / 2 + m] : conj(E[n * (n + 1) / 2 - m]);
}

/* ---- operators on raw arrays ---- */

/* P2M (kernels/laplace.h:237-252). */
static void p2m_raw(const tables_t *t, const double X[3], int n, const double *xyzq, cplx *M) {
  const int P = t->P;
  cplx Y[P * P], Yt[P * P];
  for (int b = 0; b < n; b++) {
    double d[3] = {xyzq[4 * b] - X[0], xyzq[4 * b + 1] - X[1], xyzq[4 * b + 2] - X[2]};
    double rho, al, be;
    to_sph(d, &rho, &al, &be);
    regular(t, rho, al, -be, Y, Yt);
    for (int nn = 0; nn < P; nn++)
      for (int m = 0; m <= nn; m++)
        M[nn * (nn + 1) / 2 + m] += xyzq[4 * b + 3] * Y[nn * nn + nn + m];
  }
}

/* M2M of one child into its parent (kernels/laplace.h:254-290). */
static void m2m_raw(const tables_t *t, const double Xp[3], const double Xc[3], const cplx *Mc, cplx *Mp) {
  const int P = t->P;
  cplx Y[P * P], Yt[P * P];
  double d[3] = {Xp[0] - Xc[0], Xp[1] - Xc[1], Xp[2] - Xc[2]};
  double rho, al, be;
  to_sph(d, &rho, &al, &be);
  regular(t, rho, al, -be, Y, Yt);
  for (int j = 0; j < P; j++) {
    for (int k = 0; k <= j; k++) {
      const int jk = j * j + j + k;
      cplx acc = 0;
      for (int n = 0; n <= j; n++) {
        for (int m = -n; m <= n; m++) {
          if (abs(k - m) > j - n) continue;        /* child term (j-n, k-m) must exist */
          const int nm = n * n + n + m;
          const int jnkm = (j - n) * (j - n) + j - n + k - m;
          double w = t->anm[nm] * t->anm[jnkm] / t->anm[jk];
          if (m < k) {
            /* k-m > 0: child coefficient taken directly; i^(m-|m|) = (-1)^m for m < 0 */
            double ph = (m < 0) ? sgn_pow(m) : 1.0;
            acc += Mc[(j - n) * (j - n + 1) / 2 + k - m] * ph * Y[nm] * (sgn_pow(n) * w);
          } else {
            /* k-m <= 0: conjugate of the (m-k) coefficient */
            acc += conj(Mc[(j - n) * (j - n + 1) / 2 + m - k]) * Y[nm] * (sgn_pow(k + n + m) * w);
          }
        }
      }
      Mp[j * (j + 1) / 2 + k] += acc;
    }
  }
}

/* M2L (kernels/laplace.h:292-322). */
static void m2l_raw(const tables_t *t, const double Xi[3], const double Xj[3], const double Xper[3],
                    const cplx *Mj, cplx *Li) {
  const int P = t->P;
  cplx Y[4 * P * P];
  double d[3] = {Xi[0] - Xj[0] - Xper[0], Xi[1] - Xj[1] - Xper[1], Xi[2] - Xj[2] - Xper[2]};
  double rho, al, be;
  to_sph(d, &rho, &al, &be);
  singular(t, rho, al, be, Y);
  for (int j = 0; j < P; j++) {
    for (int k = 0; k <= j; k++) {
      const int jk = j * j + j + k;
      cplx acc = 0;
      for (int n = 0; n < P; n++) {
        for (int m = -n; m <= n; m++) {
          const int nm = n * n + n + m;
          const int jnkm = (j + n) * (j + n) + j + n + m - k;
          acc += coef(Mj, n, m) * t->cjk[jk * P * P + nm] * Y[jnkm];
        }
      }
      Li[j * (j + 1) / 2 + k] += acc;
    }
  }
}

/* L2L from the parent into one child (kernels/laplace.h:324-357). */
static void l2l_raw(const tables_t *t, const double Xc[3], const double Xp[3], const cplx *Lp, cplx *Lc) {
  const int P = t->P;
  cplx Y[P * P], Yt[P * P];
  double d[3] = {Xc[0] - Xp[0], Xc[1] - Xp[1], Xc[2] - Xp[2]};
  double rho, al, be;
  to_sph(d, &rho, &al, &be);
  regular(t, rho, al, be, Y, Yt);
  for (int j = 0; j < P; j++) {
    for (int k = 0; k <= j; k++) {
      const int jk = j * j + j + k;
      cplx acc = 0;
      for (int n = j; n < P; n++) {
        for (int m = -n; m <= n; m++) {
          if (abs(m - k) > n - j) continue;        /* Y_{n-j}^{m-k} must exist */
          const int jnkm = (n - j) * (n - j) + n - j + m - k;
          const int nm = n * n + n + m;
          double w = t->anm[jnkm] * t->anm[jk] / t->anm[nm];   /* A is even in m */
          if (m < 0) {
            acc += conj(Lp[n * (n + 1) / 2 - m]) * Y[jnkm] * (sgn_pow(k) * w);
          } else {
            /* i^(m-k-|m-k|) = (-1)^(m-k) when m < k */
            double ph = (m < k) ? sgn_pow(m - k) : 1.0;
            acc += Lp[n * (n + 1) / 2 + m] * ph * Y[jnkm] * w;
          }
        }
      }
      Lc[j * (j + 1) / 2 + k] += acc;
    }
  }
}

/* L2P (kernels/laplace.h:359-388), including its +EPS offset (EPS = 1e-16). */
static void l2p_raw(const tables_t *t, const double X[3], const cplx *L, int n, const double *xyzq, double *trg) {
  const int P = t->P;
  cplx Y[P * P], Yt[P * P];
  for (int b = 0; b < n; b++) {
    double d[3] = {xyzq[4 * b] - X[0] + 1e-16, xyzq[4 * b + 1] - X[1] + 1e-16, xyzq[4 * b + 2] - X[2] + 1e-16};
    double r, th, ph;
    to_sph(d, &r, &th, &ph);
    regular(t, r, th, ph, Y, Yt);
    double pot = 0, gr = 0, gt = 0, gp = 0;
    for (int nn = 0; nn < P; nn++) {
      const cplx *Ln = L + nn * (nn + 1) / 2;
      for (int m = 0; m <= nn; m++) {
        double w = (m == 0) ? 1.0 : 2.0;
        cplx ly = Ln[m] * Y[nn * nn + nn + m];
        pot += w * creal(ly);
        gr += w * creal(ly) / r * nn;
        gt += w * creal(Ln[m] * Yt[nn * nn + nn + m]);
        gp += w * creal(ly * I) * m;
      }
    }
    /* sph2cart (kernels/laplace.h:36-45) */
    double st = sin(th), ct = cos(th), sp = sin(ph), cp = cos(ph);
    trg[4 * b] += pot;
    trg[4 * b + 1] += st * cp * gr + ct * cp / r * gt - sp / r / st * gp;
    trg[4 * b + 2] += st * sp * gr + ct * sp / r * gt + cp / r / st * gp;
    trg[4 * b + 3] += ct * gr - st / r * gt;
  }
}

/* P2P, scalar form (kernels/laplace.h:212-234). */
static void p2p_raw(int ni, const double *xi, int nj, const double *xj, const double Xper[3], double *trg) {
  for (int i = 0; i < ni; i++) {
    double pot = 0, ax = 0, ay = 0, az = 0;
    for (int j = 0; j < nj; j++) {
      double dx = xi[4 * i] - xj[4 * j] - Xper[0];
      double dy = xi[4 * i + 1] - xj[4 * j + 1] - Xper[1];
      double dz = xi[4 * i + 2] - xj[4 * j + 2] - Xper[2];
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 != 0.0) {
        double inv2 = 1.0 / r2;
        double qr = xj[4 * j + 3] * sqrt(inv2);
        double s = inv2 * qr;
        pot += qr;
        ax += dx * s;
        ay += dy * s;
        az += dz * s;
      }
    }
    trg[4 * i] += pot;
    trg[4 * i + 1] -= ax;
    trg[4 * i + 2] -= ay;
    trg[4 * i + 3] -= az;
  }
}

/* ------------------------------------------------------------------------ */
/* Bounds (include/bound_box.h:11-25): running min/max with a 1e-5 drift.    */
/* ------------------------------------------------------------------------ */
void oracle_bounds(int n, const double *xyzq, double *b) {
  if (n <= 0) {
    for (int d = 0; d < 6; d++) b[d] = 0.0;
    return;
  }
  double lo[3], hi[3];
  for (int d = 0; d < 3; d++) lo[d] = hi[d] = xyzq[d];
  for (int i = 0; i < n; i++) {
    for (int d = 0; d < 3; d++) {
      double x = xyzq[4 * i + d];
      double a = lo[d] - 1e-5, c = hi[d] + 1e-5;
      lo[d] = x < a ? x : a;
      hi[d] = x > c ? x : c;
    }
  }
  for (int d = 0; d < 3; d++) {
    b[d] = lo[d];
    b[3 + d] = hi[d];
  }
}

/* One coordinate of that recurrence with no body ever below the running value:
 * x -/+ 1e-5 applied k times, one rounded step at a time. */
double oracle_drift_seq(double x, long long k, int up) {
  volatile double v = x;
  for (long long i = 0; i < k; i++) v = up ? v + 1e-5 : v - 1e-5;
  return v;
}

/* ------------------------------------------------------------------------ */
/* Tree (include/build_tree.h).                                              */
/* ------------------------------------------------------------------------ */
typedef struct {
  double x[4];
  int ibody;
} obody;

typedef struct {
  int ibody, nbody, nnode;
  int child[8];
  double X[3];
} onode;

typedef struct {
  int iparent, ichild, nchild, ibody, nbody, level;
  double X[3], R;
} ocell;

struct oracle_run {
  int n, P, ncells, depth;
  double bounds[6];
  double box[4];
  obody *bodies;   /* tree order */
  onode *nodes;
  int nnodes, capnodes;
  ocell *cells;
  cplx *M, *L;
  int *m2l, nm2l, capm2l;
  int *p2p, np2p, capp2p;
  double *trg;     /* tree order */
};

static int new_node(oracle_run *r) {
  if (r->nnodes == r->capnodes) {
    r->capnodes = r->capnodes ? 2 * r->capnodes : 1024;
    r->nodes = (onode *)realloc(r->nodes, sizeof(onode) * r->capnodes);
  }
  return r->nnodes++;
}

/* Top-down build with a stable per-level octant partition (build_tree.h:29-108).
 * src holds the node's bodies; they are partitioned into dst and the children
 * recurse with the roles swapped.  A leaf whose data sits in the scratch array
 * copies it back, so the final order always lands in r->bodies. */
static int build_nodes(oracle_run *r, int ncrit, obody *src, obody *dst, int begin, int end,
                       const double X[3], double R0, int level, int in_scratch) {
  if (begin == end) return -1;
  int id = new_node(r);
  r->nodes[id].ibody = begin;
  r->nodes[id].nbody = end - begin;
  r->nodes[id].nnode = 1;
  for (int d = 0; d < 3; d++) r->nodes[id].X[d] = X[d];
  for (int i = 0; i < 8; i++) r->nodes[id].child[i] = -1;
  if (end - begin <= ncrit) {
    if (in_scratch) memcpy(dst + begin, src + begin, sizeof(obody) * (end - begin));
    return id;
  }
  int count[8] = {0}, offset[8];
  for (int i = begin; i < end; i++) {
    const double *x = src[i].x;
    int o = (x[0] > X[0]) + ((x[1] > X[1]) << 1) + ((x[2] > X[2]) << 2);
    count[o]++;
  }
  for (int o = 0, s = begin; o < 8; o++) {
    offset[o] = s;
    s += count[o];
  }
  int start[8];
  memcpy(start, offset, sizeof(start));
  for (int i = begin; i < end; i++) {
    const double *x = src[i].x;
    int o = (x[0] > X[0]) + ((x[1] > X[1]) << 1) + ((x[2] > X[2]) << 2);
    dst[offset[o]++] = src[i];
  }
  const double rc = R0 / (double)(1 << (level + 1));
  for (int o = 0; o < 8; o++) {
    double Xc[3];
    for (int d = 0; d < 3; d++) Xc[d] = X[d] + rc * (double)((((o >> d) & 1) * 2) - 1);
    int c = build_nodes(r, ncrit, dst, src, start[o], start[o] + count[o], Xc, R0, level + 1, !in_scratch);
    r->nodes[id].child[o] = c;
  }
  for (int o = 0; o < 8; o++)
    if (r->nodes[id].child[o] >= 0) r->nodes[id].nnode += r->nodes[r->nodes[id].child[o]].nnode;
  return id;
}

/* Flatten nodes into cells (build_tree.h:123-165): each internal cell's children
 * form one contiguous block at the next free slot, and each child's own subtree
 * is reserved right after the block, in child order. */
static void link_cells(oracle_run *r, int node, int c, int next_free, int level, int iparent, double R0) {
  onode *nd = &r->nodes[node];
  ocell *C = &r->cells[c];
  C->iparent = iparent;
  C->R = R0 / (double)(1 << level);
  for (int d = 0; d < 3; d++) C->X[d] = nd->X[d];
  C->nbody = nd->nbody;
  C->ibody = nd->ibody;
  C->level = level;
  if (level > r->depth) r->depth = level;
  if (nd->nnode == 1) {
    C->ichild = 0;
    C->nchild = 0;
    return;
  }
  int kids[8], nk = 0;
  for (int o = 0; o < 8; o++)
    if (nd->child[o] >= 0) kids[nk++] = nd->child[o];
  C->ichild = next_free;
  C->nchild = nk;
  int next = next_free + nk;
  for (int i = 0; i < nk; i++) {
    link_cells(r, kids[i], next_free + i, next, level + 1, c, R0);
    next += r->nodes[kids[i]].nnode - 1;
  }
}

static oracle_run *make_tree(int n, const double *xyzq, int ncrit, const double *bounds6) {
  oracle_run *r = (oracle_run *)calloc(1, sizeof(oracle_run));
  r->n = n;
  if (bounds6) memcpy(r->bounds, bounds6, sizeof(r->bounds));
  else oracle_bounds(n, xyzq, r->bounds);
  /* bounds2box (build_tree.h:168-180) */
  double R = 0;
  for (int d = 0; d < 3; d++) {
    r->box[d] = (r->bounds[3 + d] + r->bounds[d]) / 2;
  }
  for (int d = 0; d < 3; d++) {
    R = fmax(r->box[d] - r->bounds[d], R);
    R = fmax(r->bounds[3 + d] - r->box[d], R);
  }
  r->box[3] = R * 1.00001;
  r->bodies = (obody *)malloc(sizeof(obody) * (n > 0 ? n : 1));
  obody *scratch = (obody *)malloc(sizeof(obody) * (n > 0 ? n : 1));
  for (int i = 0; i < n; i++) {
    memcpy(r->bodies[i].x, xyzq + 4 * i, sizeof(double) * 4);
    r->bodies[i].ibody = i;
  }
  if (n > 0) {
    int root = build_nodes(r, ncrit, r->bodies, scratch, 0, n, r->box, r->box[3], 0, 0);
    r->ncells = r->nodes[root].nnode;
    r->cells = (ocell *)calloc(r->ncells, sizeof(ocell));
    link_cells(r, root, 0, 1, 0, 0, r->box[3]);
  }
  free(scratch);
  return r;
}

oracle_run *oracle_build_tree(int n, const double *xyzq, int ncrit, const double *bounds6) {
  return make_tree(n, xyzq, ncrit, bounds6);
}

/* ------------------------------------------------------------------------ */
/* Dual tree traversal (include/traversal.h:90-230).                         */
/* ------------------------------------------------------------------------ */
typedef struct {
  oracle_run *r;
  double theta;
  int nspawn;
  double Xper[3];
  int periodic_pass;   /* record only the Xperiodic == 0 pass */
} trav_t;

static void push_pair(int **v, int *n, int *cap, int a, int b) {
  if (*n == *cap) {
    *cap = *cap ? 2 * *cap : 4096;
    *v = (int *)realloc(*v, sizeof(int) * 2 * (*cap));
  }
  (*v)[2 * *n] = a;
  (*v)[2 * *n + 1] = b;
  (*n)++;
}

typedef struct {
  int *pairs, n, cap;
  double *shift;  /* per pair Xperiodic, only when images > 0 */
  int capshift;
} plist;

static void plist_push(plist *l, int a, int b, const double X[3], int with_shift) {
  int old_cap = l->cap;
  push_pair(&l->pairs, &l->n, &l->cap, a, b);
  if (with_shift) {
    if (l->cap != old_cap || !l->shift) l->shift = (double *)realloc(l->shift, sizeof(double) * 3 * l->cap);
    memcpy(l->shift + 3 * (l->n - 1), X, sizeof(double) * 3);
  }
}

typedef struct {
  trav_t base;
  plist m2l, p2p;
  int with_shift;
} travstate;

static void dual(travstate *s, int ci, int cj);

static void split(travstate *s, int ci, int cj) {
  const ocell *Ci = &s->base.r->cells[ci], *Cj = &s->base.r->cells[cj];
  if (Cj->nchild == 0) {
    for (int c = Ci->ichild; c < Ci->ichild + Ci->nchild; c++) dual(s, c, cj);
  } else if (Ci->nchild == 0) {
    for (int c = Cj->ichild; c < Cj->ichild + Cj->nchild; c++) dual(s, ci, c);
  } else if (Ci->nbody + Cj->nbody >= s->base.nspawn || ci == cj) {
    /* TraverseRange visits the full child cross product (traversal.h:180-230). */
    for (int a = Ci->ichild; a < Ci->ichild + Ci->nchild; a++)
      for (int b = Cj->ichild; b < Cj->ichild + Cj->nchild; b++) dual(s, a, b);
  } else if (Ci->R >= Cj->R) {
    for (int c = Ci->ichild; c < Ci->ichild + Ci->nchild; c++) dual(s, c, cj);
  } else {
    for (int c = Cj->ichild; c < Cj->ichild + Cj->nchild; c++) dual(s, ci, c);
  }
}

static void dual(travstate *s, int ci, int cj) {
  const ocell *Ci = &s->base.r->cells[ci], *Cj = &s->base.r->cells[cj];
  const double *Xp = s->base.Xper;
  double dx = Ci->X[0] - Cj->X[0] - Xp[0];
  double dy = Ci->X[1] - Cj->X[1] - Xp[1];
  double dz = Ci->X[2] - Cj->X[2] - Xp[2];
  double rt2 = (dx * dx + dy * dy + dz * dz) * s->base.theta * s->base.theta;
  double rr = Ci->R + Cj->R;
  if (rt2 > rr * rr * (1 - 1e-3)) {
    plist_push(&s->m2l, ci, cj, Xp, s->with_shift);
  } else if (Ci->nchild == 0 && Cj->nchild == 0) {
    if (Cj->nbody == 0) plist_push(&s->m2l, ci, cj, Xp, s->with_shift);
    else plist_push(&s->p2p, ci, cj, Xp, s->with_shift);
  } else {
    split(s, ci, cj);
  }
}

/* Counting sort of pair indices by target cell -> CSR offsets. */
static int *group_by_target(const plist *l, int ncells, int **order_out) {
  int *off = (int *)calloc(ncells + 1, sizeof(int));
  for (int p = 0; p < l->n; p++) off[l->pairs[2 * p] + 1]++;
  for (int c = 0; c < ncells; c++) off[c + 1] += off[c];
  int *fill = (int *)malloc(sizeof(int) * (ncells + 1));
  memcpy(fill, off, sizeof(int) * (ncells + 1));
  int *order = (int *)malloc(sizeof(int) * (l->n > 0 ? l->n : 1));
  for (int p = 0; p < l->n; p++) order[fill[l->pairs[2 * p]]++] = p;
  free(fill);
  *order_out = order;
  return off;
}

static const double ZERO3[3] = {0, 0, 0};

static void apply_lists(oracle_run *r, const tables_t *t, const travstate *s) {
  const int nterm = t->P * (t->P + 1) / 2;
  int *order;
  int *off = group_by_target(&s->m2l, r->ncells, &order);
#pragma omp parallel for schedule(dynamic, 4)
  for (int c = 0; c < r->ncells; c++) {
    for (int q = off[c]; q < off[c + 1]; q++) {
      int p = order[q];
      int cj = s->m2l.pairs[2 * p + 1];
      const double *Xp = s->with_shift ? s->m2l.shift + 3 * p : ZERO3;
      m2l_raw(t, r->cells[c].X, r->cells[cj].X, Xp, r->M + (size_t)cj * nterm, r->L + (size_t)c * nterm);
    }
  }
  free(off);
  free(order);
  off = group_by_target(&s->p2p, r->ncells, &order);
  double *xb = (double *)malloc(sizeof(double) * 4 * (r->n > 0 ? r->n : 1));
  for (int i = 0; i < r->n; i++) memcpy(xb + 4 * i, r->bodies[i].x, sizeof(double) * 4);
#pragma omp parallel for schedule(dynamic, 4)
  for (int c = 0; c < r->ncells; c++) {
    for (int q = off[c]; q < off[c + 1]; q++) {
      int p = order[q];
      int cj = s->p2p.pairs[2 * p + 1];
      const double *Xp = s->with_shift ? s->p2p.shift + 3 * p : ZERO3;
      const ocell *Ci = &r->cells[c], *Cj = &r->cells[cj];
      p2p_raw(Ci->nbody, xb + 4 * Ci->ibody, Cj->nbody, xb + 4 * Cj->ibody, Xp, r->trg + 4 * Ci->ibody);
    }
  }
  free(xb);
  free(off);
  free(order);
}

/* Periodic lattice of root images (traversal.h:233-287). */
static void traverse_periodic(oracle_run *r, const tables_t *t, double theta, int images, double cycle0) {
  const int nterm = t->P * (t->P + 1) / 2;
  int prange = (int)(0.5 / theta + 1);
  int neighbor = 2 * prange + 1;
  double cycle = cycle0;
  cplx *Msuper = (cplx *)malloc(sizeof(cplx) * nterm);
  memcpy(Msuper, r->M, sizeof(cplx) * nterm);   /* copy of the source root's M */
  double Xroot[3] = {r->cells[0].X[0], r->cells[0].X[1], r->cells[0].X[2]};
  cplx *Mnext = (cplx *)malloc(sizeof(cplx) * nterm);
  for (int level = 0; level < images - 1; level++) {
    for (int ix = -prange; ix <= prange; ix++)
      for (int iy = -prange; iy <= prange; iy++)
        for (int iz = -prange; iz <= prange; iz++) {
          if (ix == 0 && iy == 0 && iz == 0) continue;
          for (int cx = -prange; cx <= prange; cx++)
            for (int cy = -prange; cy <= prange; cy++)
              for (int cz = -prange; cz <= prange; cz++) {
                double Xp[3] = {(ix * neighbor + cx) * cycle, (iy * neighbor + cy) * cycle,
                                (iz * neighbor + cz) * cycle};
                m2l_raw(t, r->cells[0].X, Xroot, Xp, Msuper, r->L);
              }
        }
    /* M2M of the neighbor images into the supercell; it keeps its own M. */
    memcpy(Mnext, Msuper, sizeof(cplx) * nterm);
    for (int ix = -prange; ix <= prange; ix++)
      for (int iy = -prange; iy <= prange; iy++)
        for (int iz = -prange; iz <= prange; iz++) {
          if (ix == 0 && iy == 0 && iz == 0) continue;
          double Xc[3] = {Xroot[0] + ix * cycle, Xroot[1] + iy * cycle, Xroot[2] + iz * cycle};
          m2m_raw(t, Xroot, Xc, Msuper, Mnext);
        }
    memcpy(Msuper, Mnext, sizeof(cplx) * nterm);
    cycle *= neighbor;
  }
  free(Msuper);
  free(Mnext);
}

oracle_run *oracle_solve(int n, const double *xyzq, int P, double theta, int ncrit, int nspawn,
                         int images, double cycle, const double *bounds6, int dipole_correction) {
  const tables_t *t = tables_for(P);
  if (!t) return NULL;
  oracle_run *r = make_tree(n, xyzq, ncrit, bounds6);
  r->P = P;
  const int nterm = P * (P + 1) / 2;
  r->trg = (double *)calloc(4 * (size_t)(n > 0 ? n : 1), sizeof(double));
  if (r->ncells == 0) return r;
  r->M = (cplx *)calloc((size_t)r->ncells * nterm, sizeof(cplx));
  r->L = (cplx *)calloc((size_t)r->ncells * nterm, sizeof(cplx));
  double *xb = (double *)malloc(sizeof(double) * 4 * n);
  for (int i = 0; i < n; i++) memcpy(xb + 4 * i, r->bodies[i].x, sizeof(double) * 4);
  /* Upward pass: children sit after their parents, so a reverse sweep is post-order
   * (include/up_down_pass.h:14-22). */
  for (int c = r->ncells - 1; c >= 0; c--) {
    ocell *C = &r->cells[c];
    cplx *M = r->M + (size_t)c * nterm;
    if (C->nchild == 0) {
      p2m_raw(t, C->X, C->nbody, xb + 4 * C->ibody, M);
    } else {
      for (int k = C->ichild; k < C->ichild + C->nchild; k++)
        m2m_raw(t, C->X, r->cells[k].X, r->M + (size_t)k * nterm, M);
    }
  }
  /* Traversal (traversal.h:326-352). */
  travstate s;
  memset(&s, 0, sizeof(s));
  s.base.r = r;
  s.base.theta = theta;
  s.base.nspawn = nspawn;
  s.with_shift = images > 0;
  if (images == 0) {
    dual(&s, 0, 0);
  } else {
    for (int ix = -1; ix <= 1; ix++)
      for (int iy = -1; iy <= 1; iy++)
        for (int iz = -1; iz <= 1; iz++) {
          s.base.Xper[0] = ix * cycle;
          s.base.Xper[1] = iy * cycle;
          s.base.Xper[2] = iz * cycle;
          dual(&s, 0, 0);
        }
  }
  r->m2l = s.m2l.pairs;
  r->nm2l = s.m2l.n;
  r->p2p = s.p2p.pairs;
  r->np2p = s.p2p.n;
  apply_lists(r, t, &s);
  free(s.m2l.shift);
  free(s.p2p.shift);
  if (images > 0) traverse_periodic(r, t, theta, images, cycle);
  /* Downward pass (up_down_pass.h:25-42, 63-75): parents precede children. */
  if (r->cells[0].nchild == 0)
    l2p_raw(t, r->cells[0].X, r->L, r->cells[0].nbody, xb + 4 * r->cells[0].ibody, r->trg + 4 * r->cells[0].ibody);
  for (int c = 1; c < r->ncells; c++) {
    ocell *C = &r->cells[c];
    l2l_raw(t, C->X, r->cells[C->iparent].X, r->L + (size_t)C->iparent * nterm, r->L + (size_t)c * nterm);
    if (C->nchild == 0)
      l2p_raw(t, C->X, r->L + (size_t)c * nterm, C->nbody, xb + 4 * C->ibody, r->trg + 4 * C->ibody);
  }
  if (images > 0 && dipole_correction) {
    /* getDipole about the origin + dipoleCorrection (up_down_pass.h:78-99). */
    double dip[3] = {0, 0, 0};
    for (int i = 0; i < n; i++)
      for (int d = 0; d < 3; d++) dip[d] += xb[4 * i + d] * xb[4 * i + 3];
    double coefv = 4 * M_PI / (3 * cycle * cycle * cycle);
    double nd = dip[0] * dip[0] + dip[1] * dip[1] + dip[2] * dip[2];
    for (int i = 0; i < n; i++) {
      r->trg[4 * i] -= coefv * nd / n / xb[4 * i + 3];
      for (int d = 0; d < 3; d++) r->trg[4 * i + 1 + d] -= coefv * dip[d];
    }
  }
  free(xb);
  return r;
}

int oracle_num_cells(const oracle_run *r) { return r->ncells; }
int oracle_num_m2l(const oracle_run *r) { return r->nm2l; }
int oracle_num_p2p(const oracle_run *r) { return r->np2p; }
int oracle_depth(const oracle_run *r) { return r->depth; }
void oracle_get_bounds(const oracle_run *r, double *b) { memcpy(b, r->bounds, sizeof(r->bounds)); }

void oracle_get_trg(const oracle_run *r, double *trg) {
  for (int i = 0; i < r->n; i++) memcpy(trg + 4 * r->bodies[i].ibody, r->trg + 4 * i, sizeof(double) * 4);
}

void oracle_get_perm(const oracle_run *r, int *perm) {
  for (int i = 0; i < r->n; i++) perm[i] = r->bodies[i].ibody;
}

void oracle_get_cells(const oracle_run *r, int *ints, double *reals) {
  for (int c = 0; c < r->ncells; c++) {
    const ocell *C = &r->cells[c];
    int v[5] = {C->iparent, C->ichild, C->nchild, C->ibody, C->nbody};
    memcpy(ints + 5 * c, v, sizeof(v));
    double w[4] = {C->X[0], C->X[1], C->X[2], C->R};
    memcpy(reals + 4 * c, w, sizeof(w));
  }
}

void oracle_get_lists(const oracle_run *r, int *m2l, int *p2p) {
  if (m2l && r->nm2l) memcpy(m2l, r->m2l, sizeof(int) * 2 * r->nm2l);
  if (p2p && r->np2p) memcpy(p2p, r->p2p, sizeof(int) * 2 * r->np2p);
}

void oracle_get_expansions(const oracle_run *r, double *M, double *L) {
  size_t cnt = (size_t)r->ncells * (r->P * (r->P + 1) / 2);
  if (M && r->M) memcpy(M, r->M, sizeof(cplx) * cnt);
  if (L && r->L) memcpy(L, r->L, sizeof(cplx) * cnt);
}

void oracle_free(oracle_run *r) {
  if (!r) return;
  free(r->bodies);
  free(r->nodes);
  free(r->cells);
  free(r->M);
  free(r->L);
  free(r->m2l);
  free(r->p2p);
  free(r->trg);
  free(r);
}

/* ---- per-operator entry points ---- */
void oracle_p2m(int P, const double *X, int n, const double *xyzq, double *M) {
  p2m_raw(tables_for(P), X, n, xyzq, (cplx *)M);
}

void oracle_m2m(int P, const double *Xp, int nchild, const double *Xc, const double *Mc, double *Mp) {
  const tables_t *t = tables_for(P);
  int nterm = P * (P + 1) / 2;
  for (int c = 0; c < nchild; c++) m2m_raw(t, Xp, Xc + 3 * c, (const cplx *)Mc + (size_t)c * nterm, (cplx *)Mp);
}

void oracle_m2l(int P, const double *Xi, const double *Xj, const double *Mj, double *Li, const double *Xper) {
  m2l_raw(tables_for(P), Xi, Xj, Xper ? Xper : ZERO3, (const cplx *)Mj, (cplx *)Li);
}

void oracle_l2l(int P, const double *Xc, const double *Xp, const double *Lp, double *Lc) {
  l2l_raw(tables_for(P), Xc, Xp, (const cplx *)Lp, (cplx *)Lc);
}

void oracle_l2p(int P, const double *X, const double *L, int n, const double *xyzq, double *trg) {
  l2p_raw(tables_for(P), X, (const cplx *)L, n, xyzq, trg);
}

void oracle_p2p(int ni, const double *xi, int nj, const double *xj, const double *Xper, double *trg) {
  p2p_raw(ni, xi, nj, xj, Xper ? Xper : ZERO3, trg);
}

void oracle_direct(int ni, const double *xi, int nj, const double *xj, int images, double theta,
                   double cycle, double *trg) {
  int neighbor = (int)(2 * (0.5 / theta + 1) + 1);
  int prange = 0;
  for (int i = 0; i < images; i++) prange += (int)pow(neighbor, i);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ni; i++) {
    for (int ix = -prange; ix <= prange; ix++)
      for (int iy = -prange; iy <= prange; iy++)
        for (int iz = -prange; iz <= prange; iz++) {
          double Xp[3] = {ix * cycle, iy * cycle, iz * cycle};
          p2p_raw(1, xi + 4 * i, nj, xj, Xp, trg + 4 * i);
        }
  }
}

/* Ewald summation (ewald.h:7-197) for small systems: wave part over the waves of
 * Ewald::initWaves (ewald.h:69-95) with dft/idft (ewald.h:27-66) and the wave
 * factor of wavePart (ewald.h:160-176); real part (ewald.h:98-120) over all
 * pairs at their nearest periodic image; self term (ewald.h:150-155).  trg
 * accumulates. */
void oracle_ewald(int n, const double *xyzq, int ksize, double alpha, double sigma, double cutoff, double cycle,
                  double *trg) {
  const double scale = 2 * M_PI / cycle;
  const double coef = 2 / sigma / (cycle * cycle * cycle), coef2 = 1 / (4 * alpha * alpha);
  int nw = 0;
  for (int l = 0; l <= ksize; l++)
    for (int m = (l == 0 ? 0 : -ksize); m <= ksize; m++)
      for (int k = (l == 0 && m == 0 ? 1 : -ksize); k <= ksize; k++)
        if (l * l + m * m + k * k <= ksize * ksize) nw++;
  int *K = (int *)malloc(sizeof(int) * 3 * (nw > 0 ? nw : 1));
  double *S = (double *)calloc(2 * (nw > 0 ? nw : 1), sizeof(double));
  int w = 0;
  for (int l = 0; l <= ksize; l++)
    for (int m = (l == 0 ? 0 : -ksize); m <= ksize; m++)
      for (int k = (l == 0 && m == 0 ? 1 : -ksize); k <= ksize; k++)
        if (l * l + m * m + k * k <= ksize * ksize) {
          K[3 * w] = l;
          K[3 * w + 1] = m;
          K[3 * w + 2] = k;
          w++;
        }
#pragma omp parallel for schedule(static)
  for (int v = 0; v < nw; v++) {
    double re = 0, im = 0;
    for (int j = 0; j < n; j++) {
      double th = 0;
      for (int d = 0; d < 3; d++) th += K[3 * v + d] * xyzq[4 * j + d] * scale;
      re += xyzq[4 * j + 3] * cos(th);
      im += xyzq[4 * j + 3] * sin(th);
    }
    double k2 = 0;
    for (int d = 0; d < 3; d++) k2 += (K[3 * v + d] * scale) * (K[3 * v + d] * scale);
    const double f = coef * exp(-k2 * coef2) / k2;
    S[2 * v] = re * f;
    S[2 * v + 1] = im * f;
  }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    double t[4] = {0, 0, 0, 0};
    for (int v = 0; v < nw; v++) {
      double th = 0;
      for (int d = 0; d < 3; d++) th += K[3 * v + d] * xyzq[4 * i + d] * scale;
      const double dtmp = S[2 * v] * sin(th) - S[2 * v + 1] * cos(th);
      t[0] += S[2 * v] * cos(th) + S[2 * v + 1] * sin(th);
      for (int d = 0; d < 3; d++) t[d + 1] -= dtmp * K[3 * v + d];
    }
    trg[4 * i] += t[0];
    for (int d = 0; d < 3; d++) trg[4 * i + 1 + d] += t[d + 1] * scale;
    /* real part at the nearest image, then the self term */
    for (int j = 0; j < n; j++) {
      double dX[3];
      for (int d = 0; d < 3; d++) {
        dX[d] = xyzq[4 * i + d] - xyzq[4 * j + d];
        dX[d] -= cycle * rint(dX[d] / cycle);
      }
      const double r2 = dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2];
      if (0 < r2 && r2 < cutoff * cutoff) {
        const double r2s = r2 * alpha * alpha, rs = sqrt(r2s), inv = 1 / rs, inv2 = inv * inv;
        const double q = xyzq[4 * j + 3];
        const double dtmp = q * (M_2_SQRTPI * exp(-r2s) * inv2 + erfc(rs) * inv2 * inv) * alpha * alpha * alpha;
        trg[4 * i] += q * erfc(rs) * inv * alpha;
        for (int d = 0; d < 3; d++) trg[4 * i + 1 + d] -= dX[d] * dtmp;
      }
    }
    trg[4 * i] -= M_2_SQRTPI * xyzq[4 * i + 3] * alpha;
  }
  free(K);
  free(S);
}
