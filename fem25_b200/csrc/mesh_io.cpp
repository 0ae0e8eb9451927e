// Host-side input of the mesh files and a cache of the mesh graph.
//
// fem25_read_mesh restates RDMESHBK (mesh_utils.f:982-1165): PROJNM.nodes
// holds NELEM then one record per element (CDOMAIN, IENG(1:4)); PROJNM.mesh
// holds (NNPG, INPTYP, NORD, IITYPE, IDISP), (XLATMIN, XLONMIN, XLATMAX,
// XLONMAX) and one record per anchor (CNNPG, X, Z, XD, ZD, VARS(1:NCOEFF),
// DENS [, QP, QS when IDISP > 0]).  Records are read with Fortran
// list-directed rules: values separated by blanks, commas or line ends, a
// READ may continue onto the next lines and drops what is left of its last
// line, character values may be quoted, D exponents and r*value repeats are
// accepted.  INPTYP 1 gives (Vp, Vs), converted as the reference does:
// MU = VS**2 * DENS, LAMBDA = VP**2 * DENS - 2 MU.
//
// fem25_fazmod restates FAZMOD / VINCENTY for the model azimuth the misfit
// needs.  (fem25_graph_save / fem25_graph_load, the graph cache, live with the
// other graph entry points.)
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "fem25_internal.h"

namespace {

// list-directed record reader over a whole file
class ListReader {
 public:
  explicit ListReader(const std::string &path) {
    std::ifstream f(path);
    ok_ = (bool)f;
    std::string line;
    while (std::getline(f, line)) lines_.push_back(line);
  }
  bool ok() const { return ok_; }
  // tokens of one READ with n items; false at end of file
  bool read(int n, std::vector<std::string> *out) {
    out->clear();
    while ((int)out->size() < n) {
      if (cur_ >= lines_.size()) return false;
      split(lines_[cur_++], n, out);
    }
    return true;
  }

 private:
  void split(const std::string &s, int n, std::vector<std::string> *out) {
    size_t i = 0;
    while (i < s.size() && (int)out->size() < n) {
      while (i < s.size() && (std::isspace((unsigned char)s[i]) || s[i] == ',')) i++;
      if (i >= s.size()) break;
      std::string tok;
      if (s[i] == '\'' || s[i] == '"') {
        const char q = s[i++];
        while (i < s.size()) {
          if (s[i] == q) {
            if (i + 1 < s.size() && s[i + 1] == q) {  // doubled quote
              tok += q;
              i += 2;
              continue;
            }
            i++;
            break;
          }
          tok += s[i++];
        }
      } else {
        while (i < s.size() && !std::isspace((unsigned char)s[i]) && s[i] != ',') tok += s[i++];
      }
      // r*value repeat count
      const size_t star = tok.find('*');
      if (star != std::string::npos && star > 0 &&
          tok.find_first_not_of("0123456789") == star) {
        const int r = std::atoi(tok.substr(0, star).c_str());
        const std::string v = tok.substr(star + 1);
        for (int k = 0; k < r && (int)out->size() < n; k++) out->push_back(v);
      } else {
        out->push_back(tok);
      }
    }
  }
  std::vector<std::string> lines_;
  size_t cur_ = 0;
  bool ok_ = false;
};

bool to_double(const std::string &t, double *v) {
  std::string s = t;
  for (char &c : s)
    if (c == 'd' || c == 'D') c = 'E';
  char *end = nullptr;
  *v = std::strtod(s.c_str(), &end);
  return end && *end == '\0' && !s.empty();
}

bool to_int(const std::string &t, int *v) {
  char *end = nullptr;
  const long x = std::strtol(t.c_str(), &end, 10);
  *v = (int)x;
  return end && *end == '\0' && !t.empty();
}

}  // namespace

struct fem25_mesh_file {
  int nelem = 0, nnpg = 0, nord = 0, inptyp = 0, iitype = 0, idisp = 0, neleme = 0, nabs = 0;
  double latlon[4] = {0, 0, 0, 0};
  double xwidth = 0, zwidth = 0;
  std::vector<int> ieng;
  std::vector<char> cdomain, cnnpg;
  std::vector<double> x, z, xd, zd, ecoeff, dens, qp, qs;
};

extern "C" {

int fem25_read_mesh(const char *projnm, fem25_mesh_file **out) {
  if (!projnm || !out) return FEM25_ERR_ARG;
  *out = nullptr;
  auto err = [](int code, const char *msg) {
    std::fprintf(stderr, "fem25gpu: %s\n", msg);
    return code;
  };
  auto *f = new fem25_mesh_file();
  std::vector<std::string> t;
  {
    ListReader r(std::string(projnm) + ".nodes");
    if (!r.ok()) {
      delete f;
      return err(FEM25_ERR_ARG, "rdmeshbk: Nodes file does not exist");
    }
    if (!r.read(1, &t) || !to_int(t[0], &f->nelem) || f->nelem <= 0) {
      delete f;
      return err(FEM25_ERR_ARG, "rdmeshbk: Premature end of nodesfl");
    }
    f->cdomain.resize(f->nelem);
    f->ieng.resize(4 * (size_t)f->nelem);
    for (int e = 0; e < f->nelem; e++) {
      bool ok = r.read(5, &t) && !t[0].empty();
      for (int a = 0; ok && a < 4; a++) ok = to_int(t[1 + a], &f->ieng[4 * (size_t)e + a]);
      if (!ok) {
        delete f;
        return err(FEM25_ERR_ARG, "rdmeshbk: Premature end of nodesfl");
      }
      f->cdomain[e] = t[0][0];
      if (t[0][0] == 'E') f->neleme++;
      if (t[0][0] == 'A') f->nabs++;
    }
  }
  ListReader r(std::string(projnm) + ".mesh");
  if (!r.ok()) {
    delete f;
    return err(FEM25_ERR_ARG, "rdmeshbk: Mesh file does not exist");
  }
  bool ok = r.read(5, &t) && to_int(t[0], &f->nnpg) && to_int(t[1], &f->inptyp) &&
            to_int(t[2], &f->nord) && to_int(t[3], &f->iitype) && to_int(t[4], &f->idisp);
  ok = ok && r.read(4, &t);
  for (int k = 0; ok && k < 4; k++) ok = to_double(t[k], &f->latlon[k]);
  if (!ok || f->nnpg <= 0) {
    delete f;
    return err(FEM25_ERR_ARG, "rdmeshbk: Premature end of meshfl");
  }
  const int ncoeff = f->inptyp > 2 ? 5 : 2;
  if (ncoeff > 2 && f->idisp > 0) f->idisp = 0;  // anisotropic dispersion turned off
  const int n = f->nnpg;
  f->cnnpg.assign(2 * (size_t)n, ' ');
  f->x.resize(n);
  f->z.resize(n);
  f->xd.resize(n);
  f->zd.resize(n);
  f->ecoeff.resize((size_t)n * ncoeff);
  f->dens.resize(n);
  f->qp.assign(n, 9999.0);
  f->qs.assign(n, 9999.0);
  const int nitem = 1 + 4 + ncoeff + 1 + (f->idisp > 0 ? 2 : 0);
  std::vector<double> vars(ncoeff);
  for (int p = 0; p < n; p++) {
    ok = r.read(nitem, &t);
    double v[4];
    for (int k = 0; ok && k < 4; k++) ok = to_double(t[1 + k], &v[k]);
    for (int k = 0; ok && k < ncoeff; k++) ok = to_double(t[5 + k], &vars[k]);
    ok = ok && to_double(t[5 + ncoeff], &f->dens[p]);
    if (ok && f->idisp > 0)
      ok = to_double(t[6 + ncoeff], &f->qp[p]) && to_double(t[7 + ncoeff], &f->qs[p]);
    if (!ok) {
      delete f;
      return err(FEM25_ERR_ARG, "rdmeshbk: Premature end of meshfl");
    }
    for (int c = 0; c < 2 && c < (int)t[0].size(); c++) f->cnnpg[2 * (size_t)p + c] = t[0][c];
    f->x[p] = v[0];
    f->z[p] = v[1];
    f->xd[p] = v[2];
    f->zd[p] = v[3];
    if (f->inptyp == 1) {  // (p, s) -> lambda, mu
      const double mu = vars[1] * vars[1] * f->dens[p];
      f->ecoeff[n + (size_t)p] = mu;
      f->ecoeff[p] = vars[0] * vars[0] * f->dens[p] - 2.0 * mu;
    } else {
      for (int k = 0; k < ncoeff; k++) f->ecoeff[(size_t)k * n + p] = vars[k];
    }
    f->xwidth = std::fmax(f->xwidth, f->xd[p]);
    f->zwidth = std::fmax(f->zwidth, f->zd[p]);
  }
  *out = f;
  if (ncoeff > 2) return err(FEM25_ERR_UNSUPPORTED, "rdmeshbk: anisotropic model (INPTYP > 2)");
  if (f->iitype != 1)
    return err(FEM25_ERR_UNSUPPORTED, "rdmeshbk: IITYPE other than 1 (GLL nodes)");
  return FEM25_OK;
}

int fem25_mesh_file_get(const fem25_mesh_file *f, fem25_mesh *m, int *ints, double *reals) {
  if (!f || !m) return FEM25_ERR_ARG;
  std::memset(m, 0, sizeof(*m));
  m->nelem = f->nelem;
  m->nnpg = f->nnpg;
  m->nord = f->nord;
  m->ldisp = f->idisp > 0 ? 1 : 0;
  m->ieng = f->ieng.data();
  m->cdomain = f->cdomain.data();
  m->cnnpg = f->cnnpg.data();
  m->xlocs = f->x.data();
  m->zlocs = f->z.data();
  m->xd = f->xd.data();
  m->zd = f->zd.data();
  m->ecoeff = f->ecoeff.data();
  m->dens = f->dens.data();
  m->xwidth = f->xwidth;
  m->zwidth = f->zwidth;
  m->qp = f->qp.data();
  m->qs = f->qs.data();
  if (ints) {
    ints[0] = f->inptyp;
    ints[1] = f->iitype;
    ints[2] = f->idisp;
    ints[3] = f->neleme;
    ints[4] = f->nabs;
  }
  if (reals)
    for (int k = 0; k < 4; k++) reals[k] = f->latlon[k];
  return FEM25_OK;
}

void fem25_mesh_file_free(fem25_mesh_file *f) { delete f; }

// FAZMOD (mesh_utils.f:1166-1212) through VINCENTY (distaz.f:141-298): the
// azimuth from (XLATMIN, XLONMIN) to (XLATMAX, XLONMAX) on the WGS-84
// ellipsoid by Vincenty's inverse iteration (tolerance 1e-12 rad on lambda,
// at most 1000 iterations, the reference's pole and equator adjustments), in
// degrees in [0, 360].  Coincident points give 0.  When the iteration does not
// converge (nearly antipodal points) the reference falls back to a spherical
// routine that is not part of its repository; here that is an error.
int fem25_fazmod(double xlatmin, double xlonmin, double xlatmax, double xlonmax, double *azmod) {
  if (!azmod) return FEM25_ERR_ARG;
  const double a = 6378137.0, f = 0.0033528106647474805, pi180 = 0.017453292519943295;
  const double pi = 3.1415926535897931, hpi = 1.5707963267948966, tol = 1.0e-12, eps = 2.22e-15;
  *azmod = 0.0;
  if (std::fabs(xlonmax - xlonmin) < eps && std::fabs(xlatmax - xlatmin) < eps) return FEM25_OK;
  double phi1 = xlatmin * pi180, phi2 = xlatmax * pi180;
  // within 1e-10 rad of a pole the reference sets PHI = DSIGN(PHI,1.D0)*(HPI - 1.D-10),
  // i.e. |PHI| (HPI - 1e-10); kept as written
  if (std::fabs(hpi - std::fabs(phi1)) < 1.0e-10) phi1 = std::fabs(phi1) * (hpi - 1.0e-10);
  if (std::fabs(hpi - std::fabs(phi2)) < 1.0e-10) phi2 = std::fabs(phi2) * (hpi - 1.0e-10);
  const bool on_equator = std::fabs(phi1) < tol && std::fabs(phi2) < tol;
  const double u1 = std::atan2((1.0 - f) * std::tan(phi1), 1.0);
  const double u2 = std::atan2((1.0 - f) * std::tan(phi2), 1.0);
  const double cu1 = std::cos(u1), cu2 = std::cos(u2), su1 = std::sin(u1), su2 = std::sin(u2);
  const double dl = (xlonmax - xlonmin) * pi180;
  double lam = dl, lam0 = lam, sinl = 0.0, cosl = 0.0;
  bool done = false;
  for (int k = 0; k < 1000 && !done; k++) {
    sinl = std::sin(lam);
    cosl = std::cos(lam);
    const double t1 = cu2 * sinl, t2 = cu1 * su2 - su1 * cu2 * cosl;
    const double sins = std::sqrt(t1 * t1 + t2 * t2);
    const double coss = su1 * su2 + cu1 * cu2 * cosl;
    const double sigma = std::atan2(sins, coss);
    const double sina = cu1 * cu2 * sinl / sins;
    const double cos2a = 1.0 - sina * sina;
    const double cos2s = on_equator ? -1.0 : coss - 2.0 * su1 * su2 / cos2a;
    const double c = f / 16.0 * cos2a * (4.0 + f * (4.0 - 3.0 * cos2a));
    lam = dl + (1.0 - c) * f * sina *
                   (sigma + c * sins * (cos2s + c * coss * (-1.0 + 2.0 * cos2s * cos2s)));
    if (std::fabs(lam - lam0) < tol) {
      done = true;
    } else if (std::fabs(sins) < eps) {
      lam = pi;  // diametrically opposed
      done = true;
    }
    lam0 = lam;
  }
  if (!done) {
    std::fprintf(stderr, "fem25gpu: fazmod: Vincenty iteration did not converge\n");
    return FEM25_ERR_ARG;
  }
  // the reference takes the azimuth with the last iterate's sin/cos of lambda
  double az = std::atan2(cu2 * sinl, cu1 * su2 - su1 * cu2 * cosl) / pi180;
  if (az < 0.0) az += 360.0;
  if (az > 360.0) az -= 360.0;
  *azmod = az;
  return FEM25_OK;
}

}  // extern "C"
