// Host set-up for libfem25gpu: quadrature tables (DSHL), the mesh graph
// (GEN_GRAPH25) and the derived block-CSR / gradient pointers.  Runs once
// per mesh on the CPU; everything per (omega, py) runs on the GPU.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <unordered_map>

#include "fem25_internal.h"

namespace fem25 {

// Fortran X**N for integer N (repeated multiplication).
static double ipow(double x, int n) {
  double r = 1.0;
  for (int i = 0; i < n; i++) r = r * x;
  return r;
}

// Gauss-Lobatto-Legendre nodes and weights (the rule the reference obtains
// from gaussq.f:5 with kind=5, kpts=2): +-1 plus the roots of P'_{n-1} by
// Newton iteration on the Legendre recurrence, weights 2/(n(n-1)P_{n-1}^2).
void lobatto(int n, double *x, double *w) {
  const int N = n - 1;
  std::vector<double> xo(n);
  for (int j = 0; j < n; j++) {
    double xx = -std::cos(M_PI * (double)j / (double)N);
    for (int it = 0; it < 100; it++) {
      double p0 = 1.0, p1 = xx;
      for (int k = 2; k <= N; k++) {
        double pk = ((2.0 * k - 1.0) * xx * p1 - (k - 1.0) * p0) / (double)k;
        p0 = p1;
        p1 = pk;
      }
      double dx = (xx * p1 - p0) / ((double)(N + 1) * p1);
      xx = xx - dx;
      if (std::fabs(dx) < 1e-16) break;
    }
    xo[j] = xx;
  }
  xo[0] = -1.0;
  xo[N] = 1.0;
  for (int j = 0; j < n; j++) {
    double xx = xo[j], p0 = 1.0, p1 = xx;
    for (int k = 2; k <= N; k++) {
      double pk = ((2.0 * k - 1.0) * xx * p1 - (k - 1.0) * p0) / (double)k;
      p0 = p1;
      p1 = pk;
    }
    x[j] = xx;
    w[j] = 2.0 / ((double)(N * (N + 1)) * p1 * p1);
  }
}

// POLCOE (dshl.f:266-314): monomial coefficients of the Lagrange polynomial
static void polcoe(const double *x, const double *y, int n, double *cof, double *s) {
  for (int i = 0; i < n; i++) s[i] = cof[i] = 0.0;
  s[n - 1] = -x[0];
  for (int i = 2; i <= n; i++) {
    for (int j = n + 1 - i; j <= n - 1; j++) s[j - 1] = s[j - 1] - x[i - 1] * s[j];
    s[n - 1] = s[n - 1] - x[i - 1];
  }
  for (int j = 1; j <= n; j++) {
    double phi = (double)n;
    for (int k = n - 1; k >= 1; k--) phi = (double)k * s[k] + x[j - 1] * phi;
    double ff = y[j - 1] / phi, b = 1.0;
    for (int k = n; k >= 1; k--) {
      cof[k - 1] = cof[k - 1] + b * ff;
      b = s[k - 1] + x[j - 1] * b;
    }
  }
}

// SHAPEF (dshl.f:247-261)
static double shapef(int n, double xi, const double *cofs) {
  double v = 0.0;
  for (int i = n; i >= 2; i--) v = v + cofs[i - 1] * ipow(xi, i - 1);
  v = v + cofs[0];
  if (std::fabs(v) < 1.11e-15) v = 0.0;
  return v;
}

static void csf2d_at(double xi, double eta, double *sf, double *dsf /* [2][4] */) {
  const double EPS = 2.2204e-16;
  sf[0] = .25 * (1.0 - xi) * (1.0 - eta);
  sf[1] = .25 * (1.0 + xi) * (1.0 - eta);
  sf[2] = .25 * (1.0 + xi) * (1.0 + eta);
  sf[3] = .25 * (1.0 - xi) * (1.0 + eta);
  dsf[0] = .25 * (-1.0) * (1.0 - eta);
  dsf[1] = .25 * (1.0) * (1.0 - eta);
  dsf[2] = .25 * (1.0) * (1.0 + eta);
  dsf[3] = .25 * (-1.0) * (1.0 + eta);
  dsf[4] = .25 * (1.0 - xi) * (-1.0);
  dsf[5] = .25 * (1.0 + xi) * (-1.0);
  dsf[6] = .25 * (1.0 + xi) * (1.0);
  dsf[7] = .25 * (1.0 - xi) * (1.0);
  for (int i = 0; i < 4; i++) {
    if (std::fabs(sf[i]) < EPS) sf[i] = 0.0;
    if (std::fabs(dsf[i]) < EPS) dsf[i] = 0.0;
    if (std::fabs(dsf[4 + i]) < EPS) dsf[4 + i] = 0.0;
  }
}

void build_tables(Tables *t) {
  const double EPS = 2.11e-16;
  std::vector<double> w(kNl);
  lobatto(kNl, t->xipts, w.data());
  t->xipts[(kNl - 1) / 2] = 0.0;  // dshl.f:135 / genpts dshl.f:395
  lobatto(kNint, t->xigll, t->wts);
  t->xigll[(kNint - 1) / 2] = 0.0;  // dshl.f:145
  const double *etagll = t->xigll;
  double cofxi[kNl], cofeta[kNl], s[kNl], lagr[kNl], xil[kNint], etal[kNint];
  int ia = 0;
  for (int ieta = 1; ieta <= kNl; ieta++) {
    for (int k = 1; k <= kNl; k++) lagr[k - 1] = (k == ieta) ? 1.0 : 0.0;
    polcoe(t->xipts, lagr, kNl, cofeta, s);
    for (int intz = 1; intz <= kNint; intz++) {
      double sumd = 0.0;
      for (int k = kNl; k >= 2; k--) {
        double dk = (double)(k - 1);
        sumd = sumd + dk * cofeta[k - 1] * ipow(etagll[intz - 1], k - 2);
      }
      if (std::fabs(sumd) < EPS) sumd = 0.0;
      etal[intz - 1] = sumd;
    }
    for (int ixi = 1; ixi <= kNl; ixi++) {
      ia++;
      for (int k = 1; k <= kNl; k++) lagr[k - 1] = (k == ixi) ? 1.0 : 0.0;
      polcoe(t->xipts, lagr, kNl, cofxi, s);
      for (int intx = 1; intx <= kNint; intx++) {
        double sumd = 0.0;
        for (int k = kNl; k >= 2; k--) {
          double dk = (double)(k - 1);
          sumd = sumd + dk * cofxi[k - 1] * ipow(t->xigll[intx - 1], k - 2);
        }
        if (std::fabs(sumd) < EPS) sumd = 0.0;
        xil[intx - 1] = sumd;
      }
      for (int intz = 1; intz <= kNint; intz++)
        for (int intx = 1; intx <= kNint; intx++) {
          size_t b = 3 * ((size_t)(ia - 1) + (size_t)kNen * ((intx - 1) + (size_t)kNint * (intz - 1)));
          double sna = shapef(kNl, etagll[intz - 1], cofeta);
          double snb = shapef(kNl, t->xigll[intx - 1], cofxi);
          double v = sna * snb;
          if (std::fabs(v) < EPS) v = 0.0;
          t->shl[b + 2] = v;
          sna = shapef(kNl, etagll[intz - 1], cofeta);
          t->shl[b + 0] = sna * xil[intx - 1];
          sna = shapef(kNl, t->xigll[intx - 1], cofxi);
          t->shl[b + 1] = sna * etal[intz - 1];
          if (std::fabs(t->shl[b + 0]) < EPS) t->shl[b + 0] = 0.0;
          if (std::fabs(t->shl[b + 1]) < EPS) t->shl[b + 1] = 0.0;
        }
    }
  }
  for (int intz = 0; intz < kNint; intz++)
    for (int intx = 0; intx < kNint; intx++) {
      int q = intx + kNint * intz;
      csf2d_at(t->xigll[intx], t->xigll[intz], t->sf[q], &t->dsf[q][0][0]);
    }
}

// ---------------------------------------------------------------------------
// graph
// ---------------------------------------------------------------------------
static void csf2dnd(double xi, double eta, double *sf) {
  const double EPS = 2.2204e-16;
  sf[0] = .25 * (1.0 - xi) * (1.0 - eta);
  sf[1] = .25 * (1.0 + xi) * (1.0 - eta);
  sf[2] = .25 * (1.0 + xi) * (1.0 + eta);
  sf[3] = .25 * (1.0 - xi) * (1.0 + eta);
  for (int i = 0; i < 4; i++)
    if (std::fabs(sf[i]) < EPS) sf[i] = 0.0;
}

static inline void node_xz(const fem25_mesh *m, int e, double xi, double eta, double *x,
                           double *z) {
  double sf[4];
  csf2dnd(xi, eta, sf);
  const int *ieng = m->ieng + 4 * (size_t)e;
  double xx = 0.0, zz = 0.0;
  for (int ia = 0; ia < 4; ia++) {
    xx = xx + sf[ia] * m->xlocs[ieng[ia] - 1];
    zz = zz + sf[ia] * m->zlocs[ieng[ia] - 1];
  }
  *x = xx;
  *z = zz;
}

static inline bool on_side(int ilxi, int ileta) {
  return ilxi == 1 || ilxi == kNl || ileta == 1 || ileta == kNl;
}

static bool is_fixed(const char *c) {
  return c[0] == 'F' && (c[1] == 'L' || c[1] == 'B' || c[1] == 'R');
}

int build_graph(const fem25_mesh *m, HostGraph *g, std::string *err) {
  const double TOL = 1e-8;
  const int nelem = m->nelem;
  double pts[kNl], w[kNl];
  lobatto(kNl, pts, w);
  pts[(kNl - 1) / 2] = 0.0;
  g->nelem = nelem;

  // --- GENIEN (graph25.f:509-698): distinct element-edge nodes within TOL,
  // found with a uniform bucket grid over the anchor bounding box.
  double xmin = 1e300, xmax = -1e300, zmin = 1e300, zmax = -1e300;
  for (int p = 0; p < m->nnpg; p++) {
    xmin = std::min(xmin, m->xlocs[p]);
    xmax = std::max(xmax, m->xlocs[p]);
    zmin = std::min(zmin, m->zlocs[p]);
    zmax = std::max(zmax, m->zlocs[p]);
  }
  const int nb = 2048;
  const double hx = (xmax - xmin) / nb + 1e-6, hz = (zmax - zmin) / nb + 1e-6;
  std::unordered_map<long long, std::vector<int>> bucket;
  bucket.reserve((size_t)nelem * 8);
  std::vector<double> ux, uz;  // distinct edge nodes (insertion order)
  const int nside = 4 * (kNl - 1);
  std::vector<int> slot_node((size_t)nelem * kNen, -1);  // distinct id per edge slot
  for (int e = 0; e < nelem; e++)
    for (int ileta = 1; ileta <= kNl; ileta++)
      for (int ilxi = 1; ilxi <= kNl; ilxi++) {
        if (!on_side(ilxi, ileta)) continue;
        double x, z;
        node_xz(m, e, pts[ilxi - 1], pts[ileta - 1], &x, &z);
        long long bx = (long long)((x - xmin) / hx), bz = (long long)((z - zmin) / hz);
        int found = -1;
        for (int dx = -1; dx <= 1 && found < 0; dx++)
          for (int dz = -1; dz <= 1 && found < 0; dz++) {
            auto it = bucket.find((bx + dx) * 1000003LL + (bz + dz));
            if (it == bucket.end()) continue;
            for (int j : it->second)
              if (std::fabs(ux[j] - x) < TOL && std::fabs(uz[j] - z) < TOL) {
                found = j;
                break;
              }
          }
        if (found < 0) {
          found = (int)ux.size();
          ux.push_back(x);
          uz.push_back(z);
          bucket[bx * 1000003LL + bz].push_back(found);
        }
        slot_node[(size_t)e * kNen + (ileta - 1) * kNl + ilxi - 1] = found;
      }
  (void)nside;
  const long long nnodes = (long long)ux.size();
  // sort by x (DHPSRT2), then by z within runs of x equal to TOL (SHELL2)
  std::vector<int> ord(nnodes);
  std::iota(ord.begin(), ord.end(), 0);
  std::sort(ord.begin(), ord.end(), [&](int a, int b) {
    if (ux[a] != ux[b]) return ux[a] < ux[b];
    return uz[a] < uz[b];
  });
  auto zsort = [&](long long lo, long long hi) {  // 1-based inclusive
    std::sort(ord.begin() + (lo - 1), ord.begin() + hi, [&](int a, int b) { return uz[a] < uz[b]; });
  };
  long long jbeg = 1;
  for (long long in = 1; in <= nnodes; in++) {
    if (in + 1 == nnodes) {
      if (jbeg != nnodes) zsort(jbeg, nnodes);
      break;
    }
    if (in + 1 > nnodes) break;
    if (std::fabs(ux[ord[in]] - ux[ord[in - 1]]) > TOL) {
      if (in - jbeg + 1 > 1) zsort(jbeg, in);
      jbeg = in + 1;
    }
  }
  std::vector<int> pos(nnodes);
  for (long long i = 0; i < nnodes; i++) pos[ord[i]] = (int)i + 1;
  g->ien.assign((size_t)nelem * kNen, 0);
  int iint = (int)nnodes;
  for (int e = 0; e < nelem; e++)
    for (int iae = 0; iae < kNen; iae++) {
      int s = slot_node[(size_t)e * kNen + iae];
      g->ien[(size_t)e * kNen + iae] = (s >= 0) ? pos[s] : ++iint;
    }
  g->nnp = iint;
  const int nnp = iint;

  // --- GENID (graph25.f:315-505)
  const int LNULL = -5;
  const double TOLD = 1e-10;
  std::vector<int> id((size_t)3 * nnp, LNULL);
  for (int e = 0; e < nelem; e++) {
    if (m->cdomain[e] != 'A') continue;
    const int *ieng = m->ieng + 4 * (size_t)e;
    int icheck = 0, iav[3] = {0, 0, 0};
    for (int ia = 0; ia < 4 && icheck == 0; ia++) {
      int iloc = ieng[ia];
      if (!is_fixed(m->cnnpg + 2 * (size_t)(iloc - 1))) continue;
      iav[icheck++] = iloc;
      for (int ja = 0; ja < 4; ja++) {
        int jloc = ieng[ja];
        if (is_fixed(m->cnnpg + 2 * (size_t)(jloc - 1)) && iloc != jloc) {
          iav[icheck++] = jloc;
          if (icheck == 3) break;
        }
      }
    }
    if (icheck == 0) continue;
    for (int loop = 1; loop <= 2; loop++) {
      int ia1 = iav[0], ia2 = 0;
      double v1x = 0.0, v1z = 0.0;
      if (icheck > 1) {
        ia1 = iav[loop - 1];
        ia2 = iav[loop];
        if (ia2 == 0) break;
        v1x = m->xlocs[ia2 - 1] - m->xlocs[ia1 - 1];
        v1z = m->zlocs[ia2 - 1] - m->zlocs[ia1 - 1];
      } else if (loop == 2) {
        break;
      }
      for (int ileta = 1; ileta <= kNl; ileta++)
        for (int ilxi = 1; ilxi <= kNl; ilxi++) {
          if (!on_side(ilxi, ileta)) continue;
          int inp = g->ien[(size_t)e * kNen + (ileta - 1) * kNl + ilxi - 1];
          double x, z;
          node_xz(m, e, pts[ilxi - 1], pts[ileta - 1], &x, &z);
          bool fix;
          if (icheck == 1) {
            fix = std::fabs(x - m->xlocs[ia1 - 1]) < TOLD && std::fabs(z - m->zlocs[ia1 - 1]) < TOLD;
          } else {
            double v2x = x - m->xlocs[ia1 - 1], v2z = z - m->zlocs[ia1 - 1];
            double det = v1x * v2z - v1z * v2x;
            fix = std::fabs(det) < TOLD;
          }
          if (fix) id[3 * (size_t)(inp - 1)] = id[3 * (size_t)(inp - 1) + 1] = id[3 * (size_t)(inp - 1) + 2] = 0;
        }
    }
  }
  int idof = 0;
  for (int e = 0; e < nelem; e++)
    for (int iae = 0; iae < kNen; iae++) {
      int inp = g->ien[(size_t)e * kNen + iae];
      for (int i = 0; i < 3; i++)
        if (id[3 * (size_t)(inp - 1) + i] == LNULL) id[3 * (size_t)(inp - 1) + i] = ++idof;
    }
  g->ndof = idof;
  for (size_t i = 0; i < id.size(); i++)
    if (id[i] == LNULL) {
      *err = "graph: node without an ID";
      return FEM25_ERR_GRAPH;
    }

  // --- GENLM (graph25.f:1-37)
  g->lm.assign((size_t)3 * kNen * nelem, 0);
  for (int e = 0; e < nelem; e++)
    for (int a = 0; a < kNen; a++)
      for (int i = 0; i < 3; i++)
        g->lm[((size_t)e * kNen + a) * 3 + i] = id[3 * (size_t)(g->ien[(size_t)e * kNen + a] - 1) + i];

  // --- CSR (GENCRS_QUICK graph25.f:136-266): row = sorted distinct DOFs of
  // the elements sharing the row's node.  All three rows of a node coincide.
  std::vector<int> ecount(nnp + 1, 0);
  for (size_t k = 0; k < g->ien.size(); k++) ecount[g->ien[k]]++;
  std::vector<long long> eptr(nnp + 2, 0);
  for (int n = 1; n <= nnp; n++) eptr[n + 1] = eptr[n] + ecount[n];
  std::vector<int> elist(eptr[nnp + 1]);
  {
    std::vector<long long> cur(eptr.begin(), eptr.end());
    for (int e = 0; e < nelem; e++)
      for (int a = 0; a < kNen; a++) elist[cur[g->ien[(size_t)e * kNen + a]]++] = e;
  }
  // node of each first DOF
  std::vector<int> dofnode(g->ndof + 1, 0);
  for (int n = 1; n <= nnp; n++)
    if (id[3 * (size_t)(n - 1)] > 0) dofnode[id[3 * (size_t)(n - 1)]] = n;
  std::vector<std::vector<int>> rows(nnp + 1);
#pragma omp parallel for schedule(dynamic, 256)
  for (int n = 1; n <= nnp; n++) {
    if (id[3 * (size_t)(n - 1)] <= 0) continue;
    std::vector<int> &r = rows[n];
    for (long long k = eptr[n]; k < eptr[n + 1]; k++) {
      int e = elist[k];
      for (int j = 0; j < 3 * kNen; j++) {
        int d = g->lm[(size_t)e * 3 * kNen + j];
        if (d > 0) r.push_back(d);
      }
    }
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
  }
  g->irptr.assign(g->ndof + 1, 0);
  long long nz = 0;
  g->irptr[0] = 1;
  for (int d = 1; d <= g->ndof; d++) {
    int first = ((d - 1) / 3) * 3 + 1;
    int n = dofnode[first];
    if (n == 0) {
      *err = "graph: DOF components of a node are not consecutive";
      return FEM25_ERR_GRAPH;
    }
    nz += (long long)rows[n].size();
    if (nz > 2147483647LL) {
      *err = "graph: more than 2^31-1 nonzeros";
      return FEM25_ERR_GRAPH;
    }
    g->irptr[d] = (int)nz + 1;
  }
  g->nzero = nz;
  g->jcptr.resize(nz);
  long long o = 0;
  for (int d = 1; d <= g->ndof; d++) {
    int n = dofnode[((d - 1) / 3) * 3 + 1];
    std::memcpy(&g->jcptr[o], rows[n].data(), sizeof(int) * rows[n].size());
    o += (long long)rows[n].size();
  }

  // --- CNMESH (bielak_utils.f:934-1025)
  g->cnp.assign(g->ndof, ' ');
  for (int pass = 0; pass < 3; pass++) {
    const char dom = pass == 0 ? 'A' : pass == 1 ? 'E' : 'I';
    for (int e = 0; e < nelem; e++) {
      if (m->cdomain[e] != dom) continue;
      for (int k = 0; k < 3 * kNen; k++) {
        int d = g->lm[(size_t)e * 3 * kNen + k];
        if (d <= 0) continue;
        char &c = g->cnp[d - 1];
        if (pass == 0) c = 'A';
        else if (pass == 1) { if (c == ' ') c = 'E'; }
        else {
          if (c == ' ') c = 'I';
          else if (c == 'E') c = 'B';
          else if (c == 'A') {
            *err = "cnmesh: interior element touches an absorbing DOF";
            return FEM25_ERR_GRAPH;
          }
        }
      }
    }
  }
  for (int d = 0; d < g->ndof; d++)
    if (g->cnp[d] == ' ') {
      *err = "cnmesh: DOF not initialised";
      return FEM25_ERR_GRAPH;
    }
  return FEM25_OK;
}

int build_block_csr(int ndof, long long nzero, const int *irptr, const int *jcptr, BlockCSR *b,
                    std::string *err) {
  if (ndof % 3 != 0) {
    *err = "block csr: NDOF not a multiple of 3";
    return FEM25_ERR_PATTERN;
  }
  b->nbrow = ndof / 3;
  b->brptr.assign(b->nbrow + 1, 0);
  for (int A = 0; A < b->nbrow; A++) {
    long long s0 = irptr[3 * A] - 1, len = irptr[3 * A + 1] - irptr[3 * A];
    if (len % 3 != 0 || s0 != 9 * b->brptr[A]) {
      *err = "block csr: row length or offset not block-aligned";
      return FEM25_ERR_PATTERN;
    }
    for (int i = 1; i < 3; i++) {
      long long si = irptr[3 * A + i] - 1, li = irptr[3 * A + i + 1] - irptr[3 * A + i];
      if (li != len || si != s0 + i * len) {
        *err = "block csr: component rows differ in length";
        return FEM25_ERR_PATTERN;
      }
      for (long long k = 0; k < len; k++)
        if (jcptr[si + k] != jcptr[s0 + k]) {
          *err = "block csr: component rows differ in columns";
          return FEM25_ERR_PATTERN;
        }
    }
    for (long long k = 0; k < len; k += 3) {
      int c = jcptr[s0 + k] - 1;
      if (c % 3 != 0 || jcptr[s0 + k + 1] - 1 != c + 1 || jcptr[s0 + k + 2] - 1 != c + 2) {
        *err = "block csr: columns not in node triplets";
        return FEM25_ERR_PATTERN;
      }
    }
    b->brptr[A + 1] = b->brptr[A] + len / 3;
  }
  if (9 * b->brptr[b->nbrow] != nzero) {
    *err = "block csr: NZERO mismatch";
    return FEM25_ERR_PATTERN;
  }
  b->nblocks = b->brptr[b->nbrow];
  b->bcol.resize(b->nblocks);
  b->brow.resize(b->nblocks);
  for (int A = 0; A < b->nbrow; A++) {
    long long s0 = irptr[3 * A] - 1;
    for (long long t = 0; t < b->brptr[A + 1] - b->brptr[A]; t++) {
      b->bcol[b->brptr[A] + t] = (jcptr[s0 + 3 * t] - 1) / 3;
      b->brow[b->brptr[A] + t] = A;
    }
  }
  return FEM25_OK;
}

// GENGMASK (gengmask.f90:1-262; no mask file, LINREC and LKBDRY true, one
// partition), ELEM_WTS (gengmask.f90:758-841), GRADPTRS (gengmask.f90:962-1118)
int build_ref_grad(const fem25_mesh *m, const int *lm, RefGradSetup *r, std::string *err) {
  const int nnpg = m->nnpg, nelem = m->nelem;
  std::vector<int> cnt(nnpg, 0);
  for (int e = 0; e < nelem; e++)
    for (int a = 0; a < 4; a++) cnt[m->ieng[4 * (size_t)e + a] - 1]++;
  r->ncon = *std::max_element(cnt.begin(), cnt.end());
  r->mconn.assign((size_t)nnpg * r->ncon, 0);
  for (int e = 0; e < nelem; e++)
    for (int a = 0; a < 4; a++) {
      int p = m->ieng[4 * (size_t)e + a] - 1;
      for (int ic = 0; ic < r->ncon; ic++)
        if (r->mconn[p + (size_t)nnpg * ic] == 0) {
          r->mconn[p + (size_t)nnpg * ic] = e + 1;
          break;
        }
    }
  r->maskg.assign(nnpg, 0);
  int inpinv = 0;
  for (int p = 0; p < nnpg; p++) {
    int e = r->mconn[p];
    bool keep = !(e > 0 && m->cdomain[e - 1] != 'I');
    const char *c = m->cnnpg + 2 * (size_t)p;
    bool cls = (c[0] == 'I' && c[1] == 'I') || (c[0] == 'B' && c[1] == 'I') ||
               (c[0] == 'F' && c[1] == 'S');
    r->maskg[p] = (keep && cls) ? ++inpinv : 0;
  }
  bool lshift = false;
  for (int e = 0; e < nelem; e++)
    for (int ia = 0; ia < 4; ia++) {
      int p = m->ieng[4 * (size_t)e + ia] - 1;
      if (r->maskg[p] <= 0) continue;
      int iae = (ia == 0) ? 1 : (ia == 1) ? kNl : (ia == 2) ? kNen : kNen - kNl + 1;  // IA2IAE
      for (int i = 0; i < 3; i++)
        if (lm[((size_t)e * kNen + iae - 1) * 3 + i] <= 0) {
          r->maskg[p] = 0;
          lshift = true;
          break;
        }
    }
  if (lshift) {
    inpinv = 0;
    for (int p = 0; p < nnpg; p++)
      if (r->maskg[p] > 0) r->maskg[p] = ++inpinv;
  }
  r->nnpinv = inpinv;
  if (inpinv < 1) {
    *err = "gengmask: no points to invert at";
    return FEM25_ERR_ARG;
  }
  // ELEM_WTS
  r->elem_wts.assign(nelem, 0.0);
  std::vector<char> linit(nelem, 0);
  double wtmax = 0.0;
  for (int p = 0; p < nnpg; p++) {
    if (r->maskg[p] <= 0) continue;
    for (int ic = 0; ic < r->ncon; ic++) {
      int e = r->mconn[p + (size_t)nnpg * ic];
      if (e <= 0) break;
      if (linit[e - 1]) continue;
      double rloc = 0.0;
      for (int ia1 = 1; ia1 <= 4; ia1++) {
        int j1 = m->ieng[4 * (size_t)(e - 1) + ia1 - 1];
        int ia2 = (ia1 + 1) % 5;
        if (ia2 == 0) ia2 = 1;
        int j2 = m->ieng[4 * (size_t)(e - 1) + ia2 - 1];
        rloc = rloc + m->xlocs[j1 - 1] * m->zlocs[j2 - 1] - m->xlocs[j2 - 1] * m->zlocs[j1 - 1];
      }
      if (rloc <= 0.0) rloc = -rloc;
      rloc = rloc * 0.5;
      r->elem_wts[e - 1] = rloc;
      linit[e - 1] = 1;
      wtmax = std::max(wtmax, rloc);
    }
  }
  for (int e = 0; e < nelem; e++)
    if (r->elem_wts[e] > 0.0) r->elem_wts[e] = wtmax / r->elem_wts[e];
  // GRADPTRS
  r->jcsc.assign(inpinv + 1, 0);
  r->icsc.clear();
  r->anchor_of_col.assign(inpinv, 0);
  r->jcsc[0] = 1;
  std::vector<int> irow;
  int col = 0;
  for (int p = 0; p < nnpg; p++) {
    if (r->maskg[p] <= 0) continue;
    irow.clear();
    for (int ic = 0; ic < r->ncon; ic++) {
      int e = r->mconn[p + (size_t)nnpg * ic];
      if (e <= 0) break;
      for (int k = 0; k < 3 * kNen; k++) {
        int d = lm[(size_t)(e - 1) * 3 * kNen + k];
        if (d > 0) irow.push_back(d);
      }
    }
    std::sort(irow.begin(), irow.end());
    irow.erase(std::unique(irow.begin(), irow.end()), irow.end());
    r->icsc.insert(r->icsc.end(), irow.begin(), irow.end());
    r->anchor_of_col[col] = p;
    col++;
    r->jcsc[col] = (int)r->icsc.size() + 1;
  }
  r->nz = (long long)r->icsc.size();
  return FEM25_OK;
}

}  // namespace fem25
