/*
 * fem25 oracle -- CPU FP64 restatement of the fem25 hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  The CUDA library in fem25_b200/ is compared
 * against this file: only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * reference legs of bench.py may load it.  The product path never links it.
 *
 * Every routine restates one reference routine loop for loop (same loop
 * order, same accumulation order, no FMA contraction: build with
 * -ffp-contract=off) so that it can serve both as the numerical oracle and as
 * the timed CPU baseline.  Citations are file:line in bakerb845/fem25.
 *
 * Index conventions follow the reference: arrays that hold indices store
 * Fortran 1-based values (IENG, IEN, LM, IRPTR, JCPTR, MCONN, MASKG ...);
 * two-dimensional Fortran arrays keep their column-major layout.
 *
 * Parity status: the reference is Fortran 77/90 and no Fortran compiler is
 * available, and the reference ships no golden vectors for this path.  The
 * oracle is pinned by (i) closed-form checks of the quadrature/shape-function
 * tables, (ii) element invariants (Hermitian stiffness, rigid-body null space,
 * area), (iii) central finite differences of the misfit through a full
 * assemble + direct solve, (iv) the Bielak identity.  Parity with the
 * reference's own binary output is unpinned.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#define NDIM 3
#define NGNOD 4

/* ------------------------------------------------------------------------ */
/* mesh / graph containers (mirrored by oracle/__init__.py)                 */
/* ------------------------------------------------------------------------ */
typedef struct {
    int nelem, nnpg, nord;
    const int *ieng;        /* IENG(4,NELEM), 1-based anchor ids            */
    const char *cdomain;    /* CDOMAIN(NELEM): 'I','E','A'                   */
    const char *cnnpg;      /* CNNPG(NNPG): 2 chars per anchor               */
    const double *xlocs, *zlocs, *xd, *zd;
    const double *ecoeff;   /* ECOEFF(NNPG,2) column-major: lambda, mu      */
    const double *dens;
    double xwidth, zwidth;
    double rcoeff[2], dmax[2], kappa[2], fcent[2]; /* [0]='S' [1]='B'        */
    int ldisp;              /* LDISP: dispersive media (QP, QS, FREQ0 used)  */
    const double *qp, *qs;  /* QP(NNPG), QS(NNPG) quality factors           */
    double freq0;           /* FREQ0 reference frequency (Hz)               */
} orc_mesh;

typedef struct {
    int nnp, ndof, ncon, nen, nelem;
    long long nzero;
    int *ien;    /* IEN(NEN,NELEM) */
    int *lm;     /* LM(3,NEN,NELEM) */
    int *irptr;  /* IRPTR(NDOF+1) */
    int *jcptr;  /* JCPTR(NZERO) */
    char *cnp;   /* CNP(NDOF) */
} orc_graph;

/* ------------------------------------------------------------------------ */
/* small helpers                                                             */
/* ------------------------------------------------------------------------ */
/* Fortran X**N with integer N, evaluated as repeated multiplication. */
static double ipow(double x, int n)
{
    double r = 1.0;
    for (int i = 0; i < n; i++) r = r * x;
    return r;
}

typedef struct { double re, im; } zc;
static inline zc zmk(double a, double b) { zc z; z.re = a; z.im = b; return z; }
static inline zc zadd(zc a, zc b) { return zmk(a.re + b.re, a.im + b.im); }
static inline zc zsub(zc a, zc b) { return zmk(a.re - b.re, a.im - b.im); }
static inline zc zmul(zc a, zc b)
{
    return zmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
/* complex division, textbook form (a+ib)/(c+id) */
static inline zc zdiv(zc a, zc b)
{
    double den = b.re * b.re + b.im * b.im;
    return zmk((a.re * b.re + a.im * b.im) / den, (a.im * b.re - a.re * b.im) / den);
}

/* ------------------------------------------------------------------------ */
/* Gauss-Lobatto-Legendre rule.                                              */
/* The reference calls the netlib Golub-Welsch routine (gaussq.f:5,           */
/* kind=5, alpha=beta=0, kpts=2).  Restated from the mathematics: nodes are   */
/* +-1 and the roots of P'_{n-1}; Newton iteration on the Legendre three-term */
/* recurrence started from Chebyshev-Gauss-Lobatto nodes; weights            */
/* 2 / (n (n-1) P_{n-1}(x)^2).  Ascending order, like gausq2's sorted output. */
/* ------------------------------------------------------------------------ */
void orc_lobatto(int n, double *x, double *w)
{
    int N = n - 1;
    double *xo = (double *)malloc(sizeof(double) * n);
    for (int j = 0; j < n; j++) {
        double xx = -cos(M_PI * (double)j / (double)N);
        for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = xx, pk = xx;
            if (N == 0) pk = 1.0;
            for (int k = 2; k <= N; k++) {
                pk = ((2.0 * k - 1.0) * xx * p1 - (k - 1.0) * p0) / (double)k;
                p0 = p1; p1 = pk;
            }
            /* p1 = P_N, p0 = P_{N-1} */
            double dx = (xx * p1 - p0) / ((double)(N + 1) * p1);
            xx = xx - dx;
            if (fabs(dx) < 1e-16) break;
        }
        xo[j] = xx;
    }
    xo[0] = -1.0; xo[N] = 1.0;
    for (int j = 0; j < n; j++) {
        double xx = xo[j];
        double p0 = 1.0, p1 = xx;
        for (int k = 2; k <= N; k++) {
            double pk = ((2.0 * k - 1.0) * xx * p1 - (k - 1.0) * p0) / (double)k;
            p0 = p1; p1 = pk;
        }
        x[j] = xx;
        w[j] = 2.0 / ((double)(N * (N + 1)) * p1 * p1);
    }
    free(xo);
}

/* GENPTS (dshl.f:352-398), IITYPE=1: GLL interpolation points, midpoint 0. */
void orc_genpts(int n, double *pts)
{
    double *w = (double *)malloc(sizeof(double) * n);
    orc_lobatto(n, pts, w);
    if (n % 2 != 0) pts[(n - 1) / 2] = 0.0;
    free(w);
}

/* POLCOE (dshl.f:266-314) */
static void polcoe(const double *x, const double *y, int n, double *cof, double *s)
{
    for (int i = 0; i < n; i++) { s[i] = 0.0; cof[i] = 0.0; }
    s[n - 1] = -x[0];
    for (int i = 2; i <= n; i++) {
        for (int j = n + 1 - i; j <= n - 1; j++)
            s[j - 1] = s[j - 1] - x[i - 1] * s[j];
        s[n - 1] = s[n - 1] - x[i - 1];
    }
    for (int j = 1; j <= n; j++) {
        double phi = (double)n;
        for (int k = n - 1; k >= 1; k--) phi = (double)k * s[k] + x[j - 1] * phi;
        double ff = y[j - 1] / phi;
        double b = 1.0;
        for (int k = n; k >= 1; k--) {
            cof[k - 1] = cof[k - 1] + b * ff;
            b = s[k - 1] + x[j - 1] * b;
        }
    }
}

/* SHAPEF (dshl.f:247-261) */
static double shapef(int n, double xi, const double *cofs)
{
    double v = 0.0;
    for (int i = n; i >= 2; i--) v = v + cofs[i - 1] * ipow(xi, i - 1);
    v = v + cofs[0];
    if (fabs(v) < 1.11e-15) v = 0.0;
    return v;
}

/*
 * DSHL (dshl.f:1-243) for IITYPE=1 (GLL interpolation points).
 * xigll: XIGLL(NINT,2) column-major (points then weights); etagll identical.
 * shl:   SHL(3,NEN,NINT,NINT) column-major.
 */
void orc_dshl(int nord, int nint, double *xigll, double *shl)
{
    int nl = nord + 1, nen = nl * nl;
    const double EPS = 2.11e-16;
    double xipts[32], cofxi[32], cofeta[32], s[32], lagr[32], xil[64], etal[64];
    double *etagll = xigll; /* NINTZ == NINTX, same rule */
    orc_genpts(nl, xipts); /* gaussq + midpoint forced to 0, dshl.f:123-136 */
    orc_lobatto(nint, xigll, xigll + nint);
    if (nint % 2 != 0) xigll[(nint - 1) / 2] = 0.0; /* dshl.f:145-146 */
    int ia = 0;
    for (int ieta = 1; ieta <= nl; ieta++) {
        for (int k = 1; k <= nl; k++) lagr[k - 1] = (k == ieta) ? 1.0 : 0.0;
        polcoe(xipts, lagr, nl, cofeta, s);
        for (int intz = 1; intz <= nint; intz++) {
            double sumd = 0.0;
            for (int k = nl; k >= 2; k--) {
                double dk = (double)(k - 1);
                sumd = sumd + dk * cofeta[k - 1] * ipow(etagll[intz - 1], k - 2);
            }
            if (fabs(sumd) < EPS) sumd = 0.0;
            etal[intz - 1] = sumd;
        }
        for (int ixi = 1; ixi <= nl; ixi++) {
            ia++;
            for (int k = 1; k <= nl; k++) lagr[k - 1] = (k == ixi) ? 1.0 : 0.0;
            polcoe(xipts, lagr, nl, cofxi, s);
            for (int intx = 1; intx <= nint; intx++) {
                double sumd = 0.0;
                for (int k = nl; k >= 2; k--) {
                    double dk = (double)(k - 1);
                    sumd = sumd + dk * cofxi[k - 1] * ipow(xigll[intx - 1], k - 2);
                }
                if (fabs(sumd) < EPS) sumd = 0.0;
                xil[intx - 1] = sumd;
            }
            for (int intz = 1; intz <= nint; intz++) {
                for (int intx = 1; intx <= nint; intx++) {
                    size_t b = 3 * ((size_t)(ia - 1) + (size_t)nen * ((intx - 1) + (size_t)nint * (intz - 1)));
                    double sna = shapef(nl, etagll[intz - 1], cofeta);
                    double snb = shapef(nl, xigll[intx - 1], cofxi);
                    double v = sna * snb;
                    if (fabs(v) < EPS) v = 0.0;
                    shl[b + 2] = v;
                    sna = shapef(nl, etagll[intz - 1], cofeta);
                    shl[b + 0] = sna * xil[intx - 1];
                    sna = shapef(nl, xigll[intx - 1], cofxi);
                    shl[b + 1] = sna * etal[intz - 1];
                    if (fabs(shl[b + 0]) < EPS) shl[b + 0] = 0.0;
                    if (fabs(shl[b + 1]) < EPS) shl[b + 1] = 0.0;
                }
            }
        }
    }
}

/* CSF2D (csf2d.f:1-131), NGNOD=4 */
static int csf2d(double xi, double eta, double *sf, double *dsf /* DSF(2,4) */)
{
    const double EPS = 2.2204e-16;
    sf[0] = .25 * (1.0 - xi) * (1.0 - eta);
    sf[1] = .25 * (1.0 + xi) * (1.0 - eta);
    sf[2] = .25 * (1.0 + xi) * (1.0 + eta);
    sf[3] = .25 * (1.0 - xi) * (1.0 + eta);
    for (int i = 0; i < 4; i++) if (fabs(sf[i]) < EPS) sf[i] = 0.0;
    dsf[0 + 2 * 0] = .25 * (-1.0) * (1.0 - eta);
    dsf[0 + 2 * 1] = .25 * (1.0) * (1.0 - eta);
    dsf[0 + 2 * 2] = .25 * (1.0) * (1.0 + eta);
    dsf[0 + 2 * 3] = .25 * (-1.0) * (1.0 + eta);
    dsf[1 + 2 * 0] = .25 * (1.0 - xi) * (-1.0);
    dsf[1 + 2 * 1] = .25 * (1.0 + xi) * (-1.0);
    dsf[1 + 2 * 2] = .25 * (1.0 + xi) * (1.0);
    dsf[1 + 2 * 3] = .25 * (1.0 - xi) * (1.0);
    double s2 = 0.0, s3 = 0.0;
    for (int i = 0; i < 4; i++) {
        if (fabs(sf[i]) < EPS) sf[i] = 0.0;
        if (fabs(dsf[0 + 2 * i]) < EPS) dsf[0 + 2 * i] = 0.0;
        if (fabs(dsf[1 + 2 * i]) < EPS) dsf[1 + 2 * i] = 0.0;
        s2 = s2 + dsf[0 + 2 * i];
        s3 = s3 + dsf[1 + 2 * i];
    }
    if (fabs(s2) > EPS) return 1;
    if (fabs(s3) > EPS) return 1;
    return 0;
}

/* CSF2DND (csf2d.f:135-200), NGNOD=4 */
static void csf2dnd(double xi, double eta, double *sf)
{
    const double EPS = 2.2204e-16;
    sf[0] = .25 * (1.0 - xi) * (1.0 - eta);
    sf[1] = .25 * (1.0 + xi) * (1.0 - eta);
    sf[2] = .25 * (1.0 + xi) * (1.0 + eta);
    sf[3] = .25 * (1.0 - xi) * (1.0 + eta);
    for (int i = 0; i < 4; i++) if (fabs(sf[i]) < EPS) sf[i] = 0.0;
}

/* ------------------------------------------------------------------------ */
/* Jacobians                                                                  */
/* ------------------------------------------------------------------------ */
/* shared geometric part of CJMK_TVI / CJACCQ / DJACAB: SHG from SHL */
static void fill_shg(int nen, int nint, int intx, int intz, const double *shl,
                     double dxdxi, double dxdeta, double dzdxi, double dzdeta, double rjac,
                     double *shg)
{
    for (int iae = 0; iae < nen; iae++) {
        size_t b = 3 * ((size_t)iae + (size_t)nen * (intx + (size_t)nint * intz));
        double drnxi = shl[b + 0], drneta = shl[b + 1];
        shg[b + 2] = shl[b + 2];
        shg[b + 0] = (drnxi * dzdeta - drneta * dzdxi) / rjac;
        shg[b + 1] = -(drnxi * dxdeta - drneta * dxdxi) / rjac;
    }
}

/* CJMK_TVI (cjac.f:1-138), isotropic: DMAT(:,:,1)=lambda, DMAT(:,:,2)=mu */
static int cjmk_tvi(const orc_mesh *m, int ielem, int nen, int nint, const double *xigll,
                    const double *shl, double *det, double *rho, double *vlam, double *vmu,
                    double *shg)
{
    const double EPS = 2.22e-16;
    const int *ieng = m->ieng + 4 * ielem;
    int nnpg = m->nnpg;
    for (int intx = 0; intx < nint; intx++) {
        double xi = xigll[intx];
        for (int intz = 0; intz < nint; intz++) {
            double eta = xigll[intz];
            double sf[4], dsf[8];
            if (csf2d(xi, eta, sf, dsf)) return 1;
            double x = 0.0, z = 0.0, r = 0.0, d1 = 0.0, d2 = 0.0;
            double dxdxi = 0.0, dxdeta = 0.0, dzdxi = 0.0, dzdeta = 0.0;
            for (int ia = 0; ia < 4; ia++) {
                int iloc = ieng[ia] - 1;
                x = x + sf[ia] * m->xlocs[iloc];
                z = z + sf[ia] * m->zlocs[iloc];
                d1 = d1 + sf[ia] * m->ecoeff[iloc];
                d2 = d2 + sf[ia] * m->ecoeff[iloc + nnpg];
                r = r + sf[ia] * m->dens[iloc];
                dxdxi = dxdxi + dsf[0 + 2 * ia] * m->xlocs[iloc];
                dxdeta = dxdeta + dsf[1 + 2 * ia] * m->xlocs[iloc];
                dzdxi = dzdxi + dsf[0 + 2 * ia] * m->zlocs[iloc];
                dzdeta = dzdeta + dsf[1 + 2 * ia] * m->zlocs[iloc];
            }
            int q = intx + nint * intz;
            vlam[q] = d1; vmu[q] = d2; rho[q] = r;
            double rjac = dxdxi * dzdeta - dxdeta * dzdxi;
            det[q] = rjac;
            if (fabs(rjac) <= EPS || rjac < 0.0) return 1;
            fill_shg(nen, nint, intx, intz, shl, dxdxi, dxdeta, dzdxi, dzdeta, rjac, shg);
        }
    }
    return 0;
}

/* ZDAMPFN (cjac.f:818-921) */
static zc zdampfn(double rn, double vp, double delta, double dmax_in, double rcoeff,
                  double rkappa, double fcent, double omega)
{
    double dmax;
    if (dmax_in > 0.0) dmax = dmax_in;
    else dmax = -3.0 * vp * log(rcoeff) / (2.0 * delta);
    double d = dmax * ipow(rn / delta, 2);
    double alpha = 3.1415926535897931 * fcent * (1.0 - rn / delta);
    zc z = zadd(zmk(rkappa, 0.0), zdiv(zmk(fabs(d), 0.0), zmk(alpha, omega)));
    return zdiv(zmk(1.0, 0.0), z);
}

/* CJACCQ (cjac.f:399-581), isotropic, convolutional PML */
static int cjaccq(const orc_mesh *m, int ielem, int nen, int nint, const double *xigll,
                  const double *shl, double omega, double rcoeff, double dmax_in,
                  double rkappa, double fcent, double *det, double *rho, double *vlam,
                  double *vmu, double *shg, zc *dampx, zc *dampz)
{
    const double EPS = 2.22e-16;
    const int *ieng = m->ieng + 4 * ielem;
    int nnpg = m->nnpg;
    for (int intx = 0; intx < nint; intx++) {
        double xi = xigll[intx];
        for (int intz = 0; intz < nint; intz++) {
            double eta = xigll[intz];
            double sf[4], dsf[8];
            if (csf2d(xi, eta, sf, dsf)) return 1;
            double x = 0.0, z = 0.0, xdep = 0.0, zdep = 0.0, vel = 0.0, r = 0.0, d1 = 0.0,
                   d2 = 0.0;
            double dxdxi = 0.0, dxdeta = 0.0, dzdxi = 0.0, dzdeta = 0.0;
            for (int ia = 0; ia < 4; ia++) {
                int iloc = ieng[ia] - 1;
                x = x + sf[ia] * m->xlocs[iloc];
                z = z + sf[ia] * m->zlocs[iloc];
                d1 = d1 + sf[ia] * m->ecoeff[iloc];
                d2 = d2 + sf[ia] * m->ecoeff[iloc + nnpg];
                r = r + sf[ia] * m->dens[iloc];
                xdep = xdep + sf[ia] * m->xd[iloc];
                zdep = zdep + sf[ia] * m->zd[iloc];
                double alpha2 = (m->ecoeff[iloc] + 2.0 * m->ecoeff[iloc + nnpg]) / m->dens[iloc];
                vel = vel + sf[ia] * sqrt(alpha2);
                dxdxi = dxdxi + dsf[0 + 2 * ia] * m->xlocs[iloc];
                dxdeta = dxdeta + dsf[1 + 2 * ia] * m->xlocs[iloc];
                dzdxi = dzdxi + dsf[0 + 2 * ia] * m->zlocs[iloc];
                dzdeta = dzdeta + dsf[1 + 2 * ia] * m->zlocs[iloc];
            }
            int q = intx + nint * intz;
            vlam[q] = d1; vmu[q] = d2; rho[q] = r;
            if (xdep > EPS)
                dampx[q] = zdampfn(xdep, vel, m->xwidth, dmax_in, rcoeff, rkappa, fcent, omega);
            else
                dampx[q] = zmk(1.0, 0.0);
            if (zdep > EPS)
                dampz[q] = zdampfn(zdep, vel, m->zwidth, dmax_in, rcoeff, rkappa, fcent, omega);
            else
                dampz[q] = zmk(1.0, 0.0);
            double rjac = dxdxi * dzdeta - dxdeta * dzdxi;
            det[q] = rjac;
            if (fabs(rjac) <= EPS || rjac < 0.0) return 1;
            fill_shg(nen, nint, intx, intz, shl, dxdxi, dxdeta, dzdxi, dzdeta, rjac, shg);
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* element matrices                                                           */
/* me, ke: column-major 75x75, ME(IPE,IQE) at [ipe + nee*iqe]                 */
/* ------------------------------------------------------------------------ */
/* KM25ISOQ (estiff25.f:1-164) */
static void km25isoq(int nen, int nint, double omega, double py, const double *wts,
                     const double *vlam, const double *vmu, const double *rho,
                     const double *det, const double *shg, double *me, zc *ke)
{
    int nee = nen * NDIM;
    for (int i = 0; i < nee * nee; i++) { me[i] = 0.0; ke[i] = zmk(0.0, 0.0); }
    double wpy = omega * py, py2 = ipow(py, 2), w2 = ipow(omega, 2);
    for (int intx = 0; intx < nint; intx++) {
        for (int intz = 0; intz < nint; intz++) {
            int q = intx + nint * intz;
            double weight = wts[intx] * wts[intz] * det[q];
            double lambda = vlam[q] * weight;
            double mu = vmu[q] * weight;
            double c11 = lambda + 2.0 * mu, c12 = lambda, c13 = lambda;
            double c22 = lambda + 2.0 * mu, c23 = lambda;
            double c33 = lambda + 2.0 * mu;
            double c44 = mu, c55 = c44, c66 = c44;
            double rhow = rho[q] * weight;
            double cm1 = -w2 * (rhow - py2 * c66);
            double cm2 = -w2 * (rhow - py2 * c22);
            double cm3 = -w2 * (rhow - py2 * c44);
            for (int ibe = 0; ibe < nen; ibe++) {
                size_t bb = 3 * ((size_t)ibe + (size_t)nen * q);
                double phib = shg[bb + 2], phibx = shg[bb + 0], phibz = shg[bb + 1];
                double phibr1 = phib * cm1, phibr2 = phib * cm2, phibr3 = phib * cm3;
                double k11t1 = c11 * phibx, k11t2 = c55 * phibz;
                double k13t1 = c13 * phibz, k13t2 = c55 * phibx;
                double k22t1 = c66 * phibx, k22t2 = c44 * phibz;
                double k31t1 = c13 * phibx, k31t2 = c55 * phibz;
                double k33t1 = c33 * phibz, k33t2 = c55 * phibx;
                double k12t1 = wpy * c12 * phib, k12t2 = wpy * c66 * phibx;
                double k21t1 = wpy * c12 * phibx, k21t2 = wpy * c66 * phib;
                double k23t1 = wpy * c23 * phibz, k23t2 = wpy * c44 * phib;
                double k32t1 = wpy * c23 * phib, k32t2 = wpy * c44 * phibz;
                for (int iae = 0; iae < nen; iae++) {
                    size_t ab = 3 * ((size_t)iae + (size_t)nen * q);
                    double phia = shg[ab + 2], phiax = shg[ab + 0], phiaz = shg[ab + 1];
                    int ipe = NDIM * iae, iqe = NDIM * ibe;
#define ME(i, j) me[(i) + nee * (j)]
#define KE(i, j) ke[(i) + nee * (j)]
                    ME(ipe, iqe) = ME(ipe, iqe) + phibr1 * phia;
                    ME(ipe + 1, iqe + 1) = ME(ipe + 1, iqe + 1) + phibr2 * phia;
                    ME(ipe + 2, iqe + 2) = ME(ipe + 2, iqe + 2) + phibr3 * phia;
                    double ke11 = phiax * k11t1 + phiaz * k11t2;
                    double ke13 = phiax * k13t1 + phiaz * k13t2;
                    double ke22 = phiax * k22t1 + phiaz * k22t2;
                    double ke31 = phiaz * k31t1 + phiax * k31t2;
                    double ke33 = phiaz * k33t1 + phiax * k33t2;
                    double ke12 = phiax * k12t1 - phia * k12t2;
                    double ke21 = phia * k21t1 - phiax * k21t2;
                    double ke23 = phia * k23t1 - phiaz * k23t2;
                    double ke32 = phiaz * k32t1 - phia * k32t2;
                    KE(ipe, iqe) = zadd(KE(ipe, iqe), zmk(ke11, 0.0));
                    KE(ipe, iqe + 1) = zsub(KE(ipe, iqe + 1), zmk(0.0, ke12));
                    KE(ipe, iqe + 2) = zadd(KE(ipe, iqe + 2), zmk(ke13, 0.0));
                    KE(ipe + 1, iqe) = zadd(KE(ipe + 1, iqe), zmk(0.0, ke21));
                    KE(ipe + 1, iqe + 1) = zadd(KE(ipe + 1, iqe + 1), zmk(ke22, 0.0));
                    KE(ipe + 1, iqe + 2) = zadd(KE(ipe + 1, iqe + 2), zmk(0.0, ke23));
                    KE(ipe + 2, iqe) = zadd(KE(ipe + 2, iqe), zmk(ke31, 0.0));
                    KE(ipe + 2, iqe + 1) = zsub(KE(ipe + 2, iqe + 1), zmk(0.0, ke32));
                    KE(ipe + 2, iqe + 2) = zadd(KE(ipe + 2, iqe + 2), zmk(ke33, 0.0));
                }
            }
        }
    }
}

/* CM25ISOQ (estiff25.f:168-334) */
static void cm25isoq(int nen, int nint, double omega, double py, const double *wts,
                     const double *vlam, const double *vmu, const double *rho,
                     const double *det, const double *shg, const zc *dampx, const zc *dampz,
                     double *me, zc *ce)
{
    int nee = nen * NDIM;
    for (int i = 0; i < nee * nee; i++) { me[i] = 0.0; ce[i] = zmk(0.0, 0.0); }
    double wpy = omega * py;
    zc cwpy = zmk(0.0, wpy);
    double py2 = ipow(py, 2), w2 = ipow(omega, 2);
    for (int intx = 0; intx < nint; intx++) {
        for (int intz = 0; intz < nint; intz++) {
            int q = intx + nint * intz;
            double weight = wts[intx] * wts[intz] * det[q];
            zc ex = dampx[q], ez = dampz[q];
            double lambda = vlam[q] * weight;
            double mu = vmu[q] * weight;
            zc clam = zmk(lambda, 0.0), cmu = zmk(mu, 0.0);
            zc c11 = zadd(zadd(clam, cmu), cmu), c12 = clam, c13 = clam;
            zc c22 = zadd(zadd(clam, cmu), cmu), c23 = clam;
            zc c33 = zadd(zadd(clam, cmu), cmu);
            zc c44 = cmu, c55 = c44, c66 = c44;
            double rhow = rho[q] * weight;
            double cm1 = -w2 * (rhow - py2 * mu);
            double cm2 = -w2 * (rhow - py2 * (lambda + 2.0 * mu));
            double cm3 = -w2 * (rhow - py2 * mu);
            for (int ibe = 0; ibe < nen; ibe++) {
                size_t bb = 3 * ((size_t)ibe + (size_t)nen * q);
                double phib = shg[bb + 2];
                zc phibx = zmul(zmk(shg[bb + 0], 0.0), ex);
                zc phibz = zmul(zmk(shg[bb + 1], 0.0), ez);
                double phibr1 = cm1 * phib, phibr2 = cm2 * phib, phibr3 = cm3 * phib;
                zc k11t1 = zmul(c11, phibx), k11t2 = zmul(c55, phibz);
                zc k13t1 = zmul(c13, phibz), k13t2 = zmul(c55, phibx);
                zc k22t1 = zmul(c66, phibx), k22t2 = zmul(c44, phibz);
                zc k31t1 = zmul(c13, phibx), k31t2 = zmul(c55, phibz);
                zc k33t1 = zmul(c33, phibz), k33t2 = zmul(c55, phibx);
                zc k12t1 = zmul(zmul(cwpy, c12), zmk(phib, 0.0));
                zc k12t2 = zmul(zmul(cwpy, c66), phibx);
                zc k21t1 = zmul(zmul(cwpy, c12), phibx);
                zc k21t2 = zmul(zmul(cwpy, c66), zmk(phib, 0.0));
                zc k23t1 = zmul(zmul(cwpy, c23), phibz);
                zc k23t2 = zmul(zmul(cwpy, c44), zmk(phib, 0.0));
                zc k32t1 = zmul(zmul(cwpy, c23), zmk(phib, 0.0));
                zc k32t2 = zmul(zmul(cwpy, c44), phibz);
                for (int iae = 0; iae < nen; iae++) {
                    size_t ab = 3 * ((size_t)iae + (size_t)nen * q);
                    double phia = shg[ab + 2];
                    zc phiax = zmul(zmk(shg[ab + 0], 0.0), ex);
                    zc phiaz = zmul(zmk(shg[ab + 1], 0.0), ez);
                    int ipe = NDIM * iae, iqe = NDIM * ibe;
#define CE(i, j) ce[(i) + nee * (j)]
                    ME(ipe, iqe) = ME(ipe, iqe) + phia * phibr1;
                    ME(ipe + 1, iqe + 1) = ME(ipe + 1, iqe + 1) + phia * phibr2;
                    ME(ipe + 2, iqe + 2) = ME(ipe + 2, iqe + 2) + phia * phibr3;
                    zc ce11 = zadd(zmul(phiax, k11t1), zmul(phiaz, k11t2));
                    zc ce13 = zadd(zmul(phiax, k13t1), zmul(phiaz, k13t2));
                    zc ce22 = zadd(zmul(phiax, k22t1), zmul(phiaz, k22t2));
                    zc ce31 = zadd(zmul(phiaz, k31t1), zmul(phiax, k31t2));
                    zc ce33 = zadd(zmul(phiaz, k33t1), zmul(phiax, k33t2));
                    zc ce12 = zsub(zmul(phiax, k12t1), zmul(zmk(phia, 0.0), k12t2));
                    zc ce21 = zsub(zmul(zmk(phia, 0.0), k21t1), zmul(phiax, k21t2));
                    zc ce23 = zsub(zmul(zmk(phia, 0.0), k23t1), zmul(phiaz, k23t2));
                    zc ce32 = zsub(zmul(phiaz, k32t1), zmul(zmk(phia, 0.0), k32t2));
                    CE(ipe, iqe) = zadd(CE(ipe, iqe), ce11);
                    CE(ipe, iqe + 1) = zsub(CE(ipe, iqe + 1), ce12);
                    CE(ipe, iqe + 2) = zadd(CE(ipe, iqe + 2), ce13);
                    CE(ipe + 1, iqe) = zadd(CE(ipe + 1, iqe), ce21);
                    CE(ipe + 1, iqe + 1) = zadd(CE(ipe + 1, iqe + 1), ce22);
                    CE(ipe + 1, iqe + 2) = zadd(CE(ipe + 1, iqe + 2), ce23);
                    CE(ipe + 2, iqe) = zadd(CE(ipe + 2, iqe), ce31);
                    CE(ipe + 2, iqe + 1) = zsub(CE(ipe + 2, iqe + 1), ce32);
                    CE(ipe + 2, iqe + 2) = zadd(CE(ipe + 2, iqe + 2), ce33);
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* dispersive media (LDISP)                                                   */
/* ------------------------------------------------------------------------ */
/* VCMPLX (haskattn.f:602-646): complex velocity of Aki & Richards 5.94,
 * v (1 + ln(f/f0) / (pi Q)) - i v / (2 Q); Q = 9999 or f0 = 0 means none */
static zc vcmplx(double freq, double freq0, double v, double q)
{
    const double PI = 3.1415926535897932384626434;
    if (freq0 == 0.0 || fabs(q - 9999.0) < 1.0e-5) return zmk(v, 0.0);
    if (q == 0.0) return zmk(v, 0.0);
    double fac1 = log(freq / freq0);
    double fact = 1.0 + 1.0 / (PI * q) * fac1;
    if (fact < 0.1) fact = 0.1;
    return zmk(v * fact, -v / (2.0 * q));
}

/* Fortran Z**2 of a COMPLEX*16: Z*Z */
static inline zc zsq(zc z) { return zmul(z, z); }

/* CJKM_QUAL (cjac.f:142-278) and, for PML elements, CJCM_QUAL
 * (cjac.f:585-755): Jacobian, interpolated Vp, Vs (interpolated velocities,
 * not moduli), QP, QS and the PML stretching factors at the points */
static int cj_qual(const orc_mesh *m, int ielem, int nen, int nint, const double *xigll,
                   const double *shl, int pml, double omega, double rcoeff, double dmax_in,
                   double rkappa, double fcent, double *det, double *vp, double *vs,
                   double *qpp, double *qss, double *shg, zc *dampx, zc *dampz)
{
    const double EPS = 2.22e-16;
    const int *ieng = m->ieng + 4 * ielem;
    int nnpg = m->nnpg;
    for (int intx = 0; intx < nint; intx++) {
        double xi = xigll[intx];
        for (int intz = 0; intz < nint; intz++) {
            double eta = xigll[intz];
            double sf[4], dsf[8];
            if (csf2d(xi, eta, sf, dsf)) return 1;
            double x = 0.0, z = 0.0, xdep = 0.0, zdep = 0.0;
            double vpq = 0.0, vsq = 0.0, qpq = 0.0, qsq = 0.0;
            double dxdxi = 0.0, dxdeta = 0.0, dzdxi = 0.0, dzdeta = 0.0;
            for (int ia = 0; ia < 4; ia++) {
                int iloc = ieng[ia] - 1;
                x = x + sf[ia] * m->xlocs[iloc];
                z = z + sf[ia] * m->zlocs[iloc];
                double rlam = m->ecoeff[iloc], rmu = m->ecoeff[iloc + nnpg];
                double vpp = sqrt((rlam + 2.0 * rmu) / m->dens[iloc]);
                double vss = sqrt(rmu / m->dens[iloc]);
                vpq = vpq + sf[ia] * vpp;
                vsq = vsq + sf[ia] * vss;
                qpq = qpq + sf[ia] * m->qp[iloc];
                qsq = qsq + sf[ia] * m->qs[iloc];
                if (pml) {
                    xdep = xdep + sf[ia] * m->xd[iloc];
                    zdep = zdep + sf[ia] * m->zd[iloc];
                }
                dxdxi = dxdxi + dsf[0 + 2 * ia] * m->xlocs[iloc];
                dxdeta = dxdeta + dsf[1 + 2 * ia] * m->xlocs[iloc];
                dzdxi = dzdxi + dsf[0 + 2 * ia] * m->zlocs[iloc];
                dzdeta = dzdeta + dsf[1 + 2 * ia] * m->zlocs[iloc];
            }
            int q = intx + nint * intz;
            vp[q] = vpq; vs[q] = vsq; qpp[q] = qpq; qss[q] = qsq;
            double rjac = dxdxi * dzdeta - dxdeta * dzdxi;
            det[q] = rjac;
            if (fabs(rjac) <= EPS || rjac < 0.0) return 1;
            if (pml) {
                double vel = vpq;
                if (xdep > EPS)
                    dampx[q] = zdampfn(xdep, vel, m->xwidth, dmax_in, rcoeff, rkappa, fcent, omega);
                else
                    dampx[q] = zmk(1.0, 0.0);
                if (zdep > EPS)
                    dampz[q] = zdampfn(zdep, vel, m->zwidth, dmax_in, rcoeff, rkappa, fcent, omega);
                else
                    dampz[q] = zmk(1.0, 0.0);
            }
            fill_shg(nen, nint, intx, intz, shl, dxdxi, dxdeta, dzdxi, dzdeta, rjac, shg);
        }
    }
    return 0;
}

/* KMDAMP (estiff25.f:511-752): density-normalised element operator with
 * complex velocities; ME real, the imaginary mass part goes into KE */
static void kmdamp(int nen, int nint, double freq, double freq0, double py, const double *wts,
                   const double *vp, const double *vs, const double *qpp, const double *qss,
                   const double *det, const double *shg, double *me, zc *ke)
{
    const double TWOPI = 6.2831853071795862;
    int nee = nen * NDIM;
    for (int i = 0; i < nee * nee; i++) { me[i] = 0.0; ke[i] = zmk(0.0, 0.0); }
    double omega = TWOPI * freq, wpy = omega * py, py2 = ipow(py, 2), w2 = ipow(omega, 2);
    for (int intx = 0; intx < nint; intx++) {
        for (int intz = 0; intz < nint; intz++) {
            int q = intx + nint * intz;
            double weight = wts[intx] * wts[intz] * det[q];
            zc zvp2 = zsq(vcmplx(freq, freq0, vp[q], qpp[q]));
            zc zvs2 = zsq(vcmplx(freq, freq0, vs[q], qss[q]));
            double rvp2 = zvp2.re * weight, qvp2 = zvp2.im * weight;
            double rvs2 = zvs2.re * weight, qvs2 = zvs2.im * weight;
            double rm1 = -(w2 * weight) + w2 * py2 * rvs2, qm1 = w2 * py2 * qvs2;
            double rm2 = -(w2 * weight) + w2 * py2 * rvp2, qm2 = w2 * py2 * qvp2;
            for (int ibe = 0; ibe < nen; ibe++) {
                size_t bb = 3 * ((size_t)ibe + (size_t)nen * q);
                double phib = shg[bb + 2], phibx = shg[bb + 0], phibz = shg[bb + 1];
                double rm11t1 = rm1 * phib, qm11t1 = qm1 * phib;
                double rm22t1 = rm2 * phib, qm22t1 = qm2 * phib;
                double rk11t1 = rvp2 * phibx, qk11t1 = qvp2 * phibx;
                double rk11t2 = rvs2 * phibz, qk11t2 = qvs2 * phibz;
                double rk13t1 = rvp2 * phibz, qk13t1 = qvp2 * phibz;
                double rk13t2 = rvs2 * phibx, qk13t2 = qvs2 * phibx;
                double rk13t3 = -(2.0 * rvs2 * phibz), qk13t3 = -(2.0 * qvs2 * phibz);
                double rk22t1 = rvs2 * phibx, qk22t1 = qvs2 * phibx;
                double rk22t2 = rvs2 * phibz, qk22t2 = qvs2 * phibz;
                double rk31t1 = rvp2 * phibx, qk31t1 = qvp2 * phibx;
                double rk31t2 = rvs2 * phibz, qk31t2 = qvs2 * phibz;
                double rk31t3 = -(2.0 * rvs2 * phibx), qk31t3 = -(2.0 * qvs2 * phibx);
                double rk33t1 = rvp2 * phibz, qk33t1 = qvp2 * phibz;
                double rk33t2 = rvs2 * phibx, qk33t2 = qvs2 * phibx;
                double rk12t1 = wpy * rvp2 * phib, qk12t1 = wpy * qvp2 * phib;
                double rk12t2 = -(2.0 * wpy * rvs2 * phib), qk12t2 = -(2.0 * wpy * qvs2 * phib);
                double rk12t3 = -(wpy * rvs2 * phibx), qk12t3 = -(wpy * qvs2 * phibx);
                double rk21t1 = wpy * rvp2 * phibx, qk21t1 = wpy * qvp2 * phibx;
                double rk21t2 = -(2.0 * wpy * rvs2 * phibx), qk21t2 = -(2.0 * wpy * qvs2 * phibx);
                double rk21t3 = -(wpy * rvs2 * phib), qk21t3 = -(wpy * qvs2 * phib);
                double rk23t1 = wpy * rvp2 * phibz, qk23t1 = wpy * qvp2 * phibz;
                double rk23t2 = -(2.0 * wpy * rvs2 * phibz), qk23t2 = -(2.0 * wpy * qvs2 * phibz);
                double rk23t3 = -(wpy * rvs2 * phib), qk23t3 = -(wpy * qvs2 * phib);
                double rk32t1 = wpy * rvp2 * phib, qk32t1 = wpy * qvp2 * phib;
                double rk32t2 = -(2.0 * wpy * rvs2 * phib), qk32t2 = -(2.0 * wpy * qvs2 * phib);
                double rk32t3 = -(wpy * rvs2 * phibz), qk32t3 = -(wpy * qvs2 * phibz);
                for (int iae = 0; iae < nen; iae++) {
                    size_t ab = 3 * ((size_t)iae + (size_t)nen * q);
                    double phia = shg[ab + 2], phiax = shg[ab + 0], phiaz = shg[ab + 1];
                    int ipe = NDIM * iae, iqe = NDIM * ibe;
                    double rme11 = rm11t1 * phia, qme11 = qm11t1 * phia;
                    double rme22 = rm22t1 * phia, qme22 = qm22t1 * phia;
                    double rme33 = rme11, qme33 = qme11;
                    double rke11 = rk11t1 * phiax + rk11t2 * phiaz;
                    double qke11 = qk11t1 * phiax + qk11t2 * phiaz;
                    double rke13 = rk13t1 * phiax + rk13t2 * phiaz + rk13t3 * phiax;
                    double qke13 = qk13t1 * phiax + qk13t2 * phiaz + qk13t3 * phiax;
                    double rke22 = rk22t1 * phiax + rk22t2 * phiaz;
                    double qke22 = qk22t1 * phiax + qk22t2 * phiaz;
                    double rke31 = rk31t1 * phiaz + rk31t2 * phiax + rk31t3 * phiaz;
                    double qke31 = qk31t1 * phiaz + qk31t2 * phiax + qk31t3 * phiaz;
                    double rke33 = rk33t1 * phiaz + rk33t2 * phiax;
                    double qke33 = qk33t1 * phiaz + qk33t2 * phiax;
                    double rke12 = rk12t1 * phiax + rk12t2 * phiax + rk12t3 * phia;
                    double qke12 = qk12t1 * phiax + qk12t2 * phiax + qk12t3 * phia;
                    double rke21 = rk21t1 * phia + rk21t2 * phia + rk21t3 * phiax;
                    double qke21 = qk21t1 * phia + qk21t2 * phia + qk21t3 * phiax;
                    double rke23 = rk23t1 * phia + rk23t2 * phia + rk23t3 * phiaz;
                    double qke23 = qk23t1 * phia + qk23t2 * phia + qk23t3 * phiaz;
                    double rke32 = rk32t1 * phiaz + rk32t2 * phiaz + rk32t3 * phia;
                    double qke32 = qk32t1 * phiaz + qk32t2 * phiaz + qk32t3 * phia;
                    ME(ipe, iqe) = ME(ipe, iqe) + rme11;
                    ME(ipe + 1, iqe + 1) = ME(ipe + 1, iqe + 1) + rme22;
                    ME(ipe + 2, iqe + 2) = ME(ipe + 2, iqe + 2) + rme33;
                    KE(ipe, iqe) = zadd(KE(ipe, iqe), zmk(rke11, qke11 + qme11));
                    KE(ipe + 1, iqe + 1) = zadd(KE(ipe + 1, iqe + 1), zmk(rke22, qke22 + qme22));
                    KE(ipe + 2, iqe + 2) = zadd(KE(ipe + 2, iqe + 2), zmk(rke33, qke33 + qme33));
                    KE(ipe, iqe + 2) = zadd(KE(ipe, iqe + 2), zmk(rke13, qke13));
                    KE(ipe + 2, iqe) = zadd(KE(ipe + 2, iqe), zmk(rke31, qke31));
                    KE(ipe, iqe + 1) = zsub(KE(ipe, iqe + 1), zmk(-qke12, rke12));
                    KE(ipe + 1, iqe) = zadd(KE(ipe + 1, iqe), zmk(-qke21, rke21));
                    KE(ipe + 1, iqe + 2) = zadd(KE(ipe + 1, iqe + 2), zmk(-qke23, rke23));
                    KE(ipe + 2, iqe + 1) = zsub(KE(ipe + 2, iqe + 1), zmk(-qke32, rke32));
                }
            }
        }
    }
}

static inline zc zneg(zc a) { return zmk(-a.re, -a.im); }

/* CMDAMP (estiff25.f:756-961): PML version of KMDAMP with the stretched
 * derivatives d/dx EX, d/dz EZ and complex arithmetic throughout */
static void cmdamp(int nen, int nint, double freq, double freq0, double py, const double *wts,
                   const double *vp, const double *vs, const double *qpp, const double *qss,
                   const double *det, const double *shg, const zc *dampx, const zc *dampz,
                   double *me, zc *ce)
{
    const double TWOPI = 6.2831853071795862;
    int nee = nen * NDIM;
    for (int i = 0; i < nee * nee; i++) { me[i] = 0.0; ce[i] = zmk(0.0, 0.0); }
    double omega = TWOPI * freq, wpy = omega * py;
    zc cwpy = zmk(0.0, wpy), ztwo = zmk(2.0, 0.0);
    double py2 = ipow(py, 2), w2 = ipow(omega, 2);
    for (int intx = 0; intx < nint; intx++) {
        for (int intz = 0; intz < nint; intz++) {
            int q = intx + nint * intz;
            double weight = wts[intx] * wts[intz] * det[q];
            zc ex = dampx[q], ez = dampz[q];
            zc zvp2 = zmul(zsq(vcmplx(freq, freq0, vp[q], qpp[q])), zmk(weight, 0.0));
            zc zvs2 = zmul(zsq(vcmplx(freq, freq0, vs[q], qss[q])), zmk(weight, 0.0));
            double rvp2 = zvp2.re, qvp2 = zvp2.im, rvs2 = zvs2.re, qvs2 = zvs2.im;
            double rm1 = -(w2 * weight) + w2 * py2 * rvs2, qm1 = w2 * py2 * qvs2;
            double rm2 = -(w2 * weight) + w2 * py2 * rvp2, qm2 = w2 * py2 * qvp2;
            for (int ibe = 0; ibe < nen; ibe++) {
                size_t bb = 3 * ((size_t)ibe + (size_t)nen * q);
                double phib = shg[bb + 2];
                zc phibx = zmul(zmk(shg[bb + 0], 0.0), ex);
                zc phibz = zmul(zmk(shg[bb + 1], 0.0), ez);
                zc cphib = zmk(phib, 0.0);
                double rm11t1 = rm1 * phib, qm11t1 = qm1 * phib;
                double rm22t1 = rm2 * phib, qm22t1 = qm2 * phib;
                zc ce11t1 = zmul(zvp2, phibx), ce11t2 = zmul(zvs2, phibz);
                zc ce13t1 = zmul(zvp2, phibz), ce13t2 = zmul(zvs2, phibx);
                zc ce13t3 = zneg(zmul(zmul(ztwo, zvs2), phibz));
                zc ce22t1 = zmul(zvs2, phibx), ce22t2 = zmul(zvs2, phibz);
                zc ce31t1 = zmul(zvp2, phibx), ce31t2 = zmul(zvs2, phibz);
                zc ce31t3 = zneg(zmul(zmul(ztwo, zvs2), phibx));
                zc ce33t1 = zmul(zvp2, phibz), ce33t2 = zmul(zvs2, phibx);
                zc ce12t1 = zmul(zmul(cwpy, zvp2), cphib);
                zc ce12t2 = zneg(zmul(zmul(zmul(ztwo, cwpy), zvs2), cphib));
                zc ce12t3 = zneg(zmul(zmul(cwpy, zvs2), phibx));
                zc ce21t1 = zmul(zmul(cwpy, zvp2), phibx);
                zc ce21t2 = zneg(zmul(zmul(zmul(ztwo, cwpy), zvs2), phibx));
                zc ce21t3 = zneg(zmul(zmul(cwpy, zvs2), cphib));
                zc ce23t1 = zmul(zmul(cwpy, zvp2), phibz);
                zc ce23t2 = zneg(zmul(zmul(zmul(ztwo, cwpy), zvs2), phibz));
                zc ce23t3 = zneg(zmul(zmul(cwpy, zvs2), cphib));
                zc ce32t1 = zmul(zmul(cwpy, zvp2), cphib);
                zc ce32t2 = zneg(zmul(zmul(zmul(ztwo, cwpy), zvs2), cphib));
                zc ce32t3 = zneg(zmul(zmul(cwpy, zvs2), phibz));
                for (int iae = 0; iae < nen; iae++) {
                    size_t ab = 3 * ((size_t)iae + (size_t)nen * q);
                    double phia = shg[ab + 2];
                    zc phiax = zmul(zmk(shg[ab + 0], 0.0), ex);
                    zc phiaz = zmul(zmk(shg[ab + 1], 0.0), ez);
                    zc cphia = zmk(phia, 0.0);
                    int ipe = NDIM * iae, iqe = NDIM * ibe;
                    double rme11 = rm11t1 * phia, qme11 = qm11t1 * phia;
                    double rme22 = rm22t1 * phia, qme22 = qm22t1 * phia;
                    double rme33 = rme11, qme33 = qme11;
                    zc ce11 = zadd(zmul(ce11t1, phiax), zmul(ce11t2, phiaz));
                    zc ce13 = zadd(zadd(zmul(ce13t1, phiax), zmul(ce13t2, phiaz)), zmul(ce13t3, phiax));
                    zc ce22 = zadd(zmul(ce22t1, phiax), zmul(ce22t2, phiaz));
                    zc ce31 = zadd(zadd(zmul(ce31t1, phiaz), zmul(ce31t2, phiax)), zmul(ce31t3, phiaz));
                    zc ce33 = zadd(zmul(ce33t1, phiaz), zmul(ce33t2, phiax));
                    zc ce12 = zadd(zadd(zmul(ce12t1, phiax), zmul(ce12t2, phiax)), zmul(ce12t3, cphia));
                    zc ce21 = zadd(zadd(zmul(ce21t1, cphia), zmul(ce21t2, cphia)), zmul(ce21t3, phiax));
                    zc ce23 = zadd(zadd(zmul(ce23t1, cphia), zmul(ce23t2, cphia)), zmul(ce23t3, phiaz));
                    zc ce32 = zadd(zadd(zmul(ce32t1, phiaz), zmul(ce32t2, phiaz)), zmul(ce32t3, cphia));
                    ME(ipe, iqe) = ME(ipe, iqe) + rme11;
                    ME(ipe + 1, iqe + 1) = ME(ipe + 1, iqe + 1) + rme22;
                    ME(ipe + 2, iqe + 2) = ME(ipe + 2, iqe + 2) + rme33;
                    CE(ipe, iqe) = zadd(zadd(CE(ipe, iqe), ce11), zmk(0.0, qme11));
                    CE(ipe, iqe + 1) = zsub(CE(ipe, iqe + 1), ce12);
                    CE(ipe, iqe + 2) = zadd(CE(ipe, iqe + 2), ce13);
                    CE(ipe + 1, iqe) = zadd(CE(ipe + 1, iqe), ce21);
                    CE(ipe + 1, iqe + 1) = zadd(zadd(CE(ipe + 1, iqe + 1), ce22), zmk(0.0, qme22));
                    CE(ipe + 1, iqe + 2) = zadd(CE(ipe + 1, iqe + 2), ce23);
                    CE(ipe + 2, iqe) = zadd(CE(ipe + 2, iqe), ce31);
                    CE(ipe + 2, iqe + 1) = zsub(CE(ipe + 2, iqe + 1), ce32);
                    CE(ipe + 2, iqe + 2) = zadd(zadd(CE(ipe + 2, iqe + 2), ce33), zmk(0.0, qme33));
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* element workspace                                                          */
/* ------------------------------------------------------------------------ */
typedef struct {
    int nord, nl, nen, nee, nint, nq;
    double *xigll, *shl, *shg, *det, *rho, *vlam, *vmu, *me;
    double *vp, *vs, *qpp, *qss;   /* dispersive media */
    zc *ke, *dampx, *dampz;
} orc_ws;

static void ws_init(orc_ws *w, int nord)
{
    w->nord = nord; w->nl = nord + 1; w->nen = w->nl * w->nl; w->nee = 3 * w->nen;
    w->nint = 2 * nord + 2 + 3; /* asmble.f90:110-112 */
    w->nq = w->nint * w->nint;
    w->xigll = (double *)malloc(sizeof(double) * 2 * w->nint);
    w->shl = (double *)malloc(sizeof(double) * 3 * w->nen * w->nq);
    w->shg = (double *)malloc(sizeof(double) * 3 * w->nen * w->nq);
    w->det = (double *)malloc(sizeof(double) * w->nq);
    w->rho = (double *)malloc(sizeof(double) * w->nq);
    w->vlam = (double *)malloc(sizeof(double) * w->nq);
    w->vmu = (double *)malloc(sizeof(double) * w->nq);
    w->vp = (double *)malloc(sizeof(double) * w->nq);
    w->vs = (double *)malloc(sizeof(double) * w->nq);
    w->qpp = (double *)malloc(sizeof(double) * w->nq);
    w->qss = (double *)malloc(sizeof(double) * w->nq);
    w->me = (double *)malloc(sizeof(double) * w->nee * w->nee);
    w->ke = (zc *)malloc(sizeof(zc) * w->nee * w->nee);
    w->dampx = (zc *)malloc(sizeof(zc) * w->nq);
    w->dampz = (zc *)malloc(sizeof(zc) * w->nq);
    orc_dshl(nord, w->nint, w->xigll, w->shl);
}

static void ws_free(orc_ws *w)
{
    free(w->xigll); free(w->shl); free(w->shg); free(w->det); free(w->rho);
    free(w->vlam); free(w->vmu); free(w->me); free(w->ke); free(w->dampx); free(w->dampz);
    free(w->vp); free(w->vs); free(w->qpp); free(w->qss);
}

/* element matrices of one element as ASMBLE_DRIVER builds them
 * (asmble.f90:140-204), isotropic media, dispersive when m->ldisp */
static int element_mats(const orc_mesh *m, orc_ws *w, int ielem, char cftype, double freq,
                        double py)
{
    const double TWOPI = 6.2831853071795862;
    double omega = TWOPI * freq;
    int k = (cftype == 'S') ? 0 : 1;
    const double *wts = w->xigll + w->nint;
    if (m->ldisp) {
        int pml = m->cdomain[ielem] == 'A';
        if (cj_qual(m, ielem, w->nen, w->nint, w->xigll, w->shl, pml, omega, m->rcoeff[k],
                    m->dmax[k], m->kappa[k], m->fcent[k], w->det, w->vp, w->vs, w->qpp, w->qss,
                    w->shg, w->dampx, w->dampz))
            return 1;
        if (!pml)
            kmdamp(w->nen, w->nint, freq, m->freq0, py, wts, w->vp, w->vs, w->qpp, w->qss, w->det,
                   w->shg, w->me, w->ke);
        else
            cmdamp(w->nen, w->nint, freq, m->freq0, py, wts, w->vp, w->vs, w->qpp, w->qss, w->det,
                   w->shg, w->dampx, w->dampz, w->me, w->ke);
        return 0;
    }
    if (m->cdomain[ielem] != 'A') {
        if (cjmk_tvi(m, ielem, w->nen, w->nint, w->xigll, w->shl, w->det, w->rho, w->vlam,
                     w->vmu, w->shg))
            return 1;
        km25isoq(w->nen, w->nint, omega, py, wts, w->vlam, w->vmu, w->rho, w->det, w->shg,
                 w->me, w->ke);
    } else {
        if (cjaccq(m, ielem, w->nen, w->nint, w->xigll, w->shl, omega, m->rcoeff[k], m->dmax[k],
                   m->kappa[k], m->fcent[k], w->det, w->rho, w->vlam, w->vmu, w->shg, w->dampx,
                   w->dampz))
            return 1;
        cm25isoq(w->nen, w->nint, omega, py, wts, w->vlam, w->vmu, w->rho, w->det, w->shg,
                 w->dampx, w->dampz, w->me, w->ke);
    }
    return 0;
}

/* exported: element matrix of one element (ME real, CE complex interleaved) */
int orc_element_matrix(const orc_mesh *m, int ielem, char cftype, double freq, double py,
                       double *me, double *ce)
{
    orc_ws w;
    ws_init(&w, m->nord);
    int ierr = element_mats(m, &w, ielem, cftype, freq, py);
    if (!ierr) {
        memcpy(me, w.me, sizeof(double) * w.nee * w.nee);
        memcpy(ce, w.ke, sizeof(zc) * w.nee * w.nee);
    }
    ws_free(&w);
    return ierr;
}

/* exported: quadrature tables */
void orc_tables(int nord, double *xigll, double *shl)
{
    int nint = 2 * nord + 2 + 3;
    orc_dshl(nord, nint, xigll, shl);
}

/* IBSECT (sort.f:1006-1042) */
static int ibsect(int n, int ix, const int *ivec)
{
    if (ix == ivec[0]) return 1;
    if (ix == ivec[n - 1]) return n;
    int jl = 0, ju = n + 1;
    while (ju - jl > 1) {
        int jm = (ju + jl) / 2;
        if ((ivec[n - 1] >= ivec[0]) == (ix >= ivec[jm - 1])) jl = jm;
        else ju = jm;
    }
    if (jl >= 1 && ix == ivec[jl - 1]) return jl;
    return -1;
}

/*
 * ASMBLE_DRIVER + ASMBLE_CDIST (asmble.f90:1-314), single process
 * (MYDOFS = 1..NDOF, local CSR = global CSR, MYELEM = 1..NELEM).
 * Elements [elo, ehi) only (full assembly: 0, nelem); the outputs are
 * accumulated, so the caller zeroes them once (asmble.f90:137).
 *   csr128: complex128 sum in FP64 of the element contributions, element order
 *   csr64:  the reference's own COMPLEX*8 accumulation: each FP64 ME+CE entry
 *           is rounded to FP32 and added in FP32 (asmble.f90:302-305)
 * Either output may be NULL.
 */
int orc_asmble(const orc_mesh *m, const int *lm, const int *irptr, const int *jcptr, int ndof,
               char cftype, double freq, double py, int elo, int ehi, double *csr128,
               float *csr64)
{
    orc_ws w;
    ws_init(&w, m->nord);
    int nen = w.nen, nee = w.nee;
    int ierr = 0;
    for (int ielem = elo; ielem < ehi && !ierr; ielem++) {
        ierr = element_mats(m, &w, ielem, cftype, freq, py);
        if (ierr) break;
        const int *lme = lm + (size_t)3 * nen * ielem;
        for (int ipe = 0; ipe < nee; ipe++) {
            int idof = lme[ipe];
            if (idof == 0) continue;
            /* IBSECT2 on MYDOFS = identity */
            int jbeg = irptr[idof - 1], jend = irptr[idof] - 1;
            int nvar = jend - jbeg + 1;
            for (int iqe = 0; iqe < nee; iqe++) {
                int jdof = lme[iqe];
                if (jdof == 0) continue;
                int indx = ibsect(nvar, jdof, jcptr + (jbeg - 1));
                if (indx <= 0) { ierr = 2; break; }
                size_t iz = (size_t)(jbeg - 1 + indx - 1);
                double r1 = w.me[ipe + nee * iqe] + w.ke[ipe + nee * iqe].re;
                double q1 = w.ke[ipe + nee * iqe].im;
                if (csr128) {
                    csr128[2 * iz] = csr128[2 * iz] + r1;
                    csr128[2 * iz + 1] = csr128[2 * iz + 1] + q1;
                }
                if (csr64) {
                    float fr = (float)r1, fq = (float)q1;
                    csr64[2 * iz] = csr64[2 * iz] + fr;
                    csr64[2 * iz + 1] = csr64[2 * iz + 1] + fq;
                }
            }
            if (ierr) break;
        }
    }
    ws_free(&w);
    return ierr;
}

/*
 * Row-restricted assembly (ASMBLE_DRIVER / ASMBLE_CDIST, asmble.f90:140-305,
 * for a subset of rows): rowoff[dof-1] >= 0 selects a 1-based DOF row and
 * gives the compact offset of its first entry in out128 / out64 (either may
 * be NULL); the row's entries follow in JCPTR order.  Same arithmetic and
 * element order as orc_asmble (FP64 sums and the reference's FP32
 * cast-then-add), so the selected rows equal the full assembly's bit for
 * bit; only the elements touching a selected row are integrated, which
 * makes spot checks of full-size systems cheap.
 */
int orc_asmble_rows(const orc_mesh *m, const int *lm, const int *irptr, const int *jcptr,
                    int ndof, const long long *rowoff, char cftype, double freq, double py,
                    double *out128, float *out64)
{
    orc_ws w;
    ws_init(&w, m->nord);
    int nen = w.nen, nee = w.nee, ierr = 0;
    for (int ielem = 0; ielem < m->nelem && !ierr; ielem++) {
        const int *lme = lm + (size_t)3 * nen * ielem;
        int touch = 0;
        for (int ipe = 0; ipe < nee; ipe++)
            if (lme[ipe] > 0 && lme[ipe] <= ndof && rowoff[lme[ipe] - 1] >= 0) { touch = 1; break; }
        if (!touch) continue;
        ierr = element_mats(m, &w, ielem, cftype, freq, py);
        if (ierr) break;
        for (int ipe = 0; ipe < nee; ipe++) {
            int idof = lme[ipe];
            if (idof == 0 || rowoff[idof - 1] < 0) continue;
            int jbeg = irptr[idof - 1], jend = irptr[idof] - 1;
            int nvar = jend - jbeg + 1;
            for (int iqe = 0; iqe < nee; iqe++) {
                int jdof = lme[iqe];
                if (jdof == 0) continue;
                int indx = ibsect(nvar, jdof, jcptr + (jbeg - 1));
                if (indx <= 0) { ierr = 2; break; }
                size_t iz = (size_t)(rowoff[idof - 1] + indx - 1);
                double r1 = w.me[ipe + nee * iqe] + w.ke[ipe + nee * iqe].re;
                double q1 = w.ke[ipe + nee * iqe].im;
                if (out128) {
                    out128[2 * iz] = out128[2 * iz] + r1;
                    out128[2 * iz + 1] = out128[2 * iz + 1] + q1;
                }
                if (out64) {
                    float fr = (float)r1, fq = (float)q1;
                    out64[2 * iz] = out64[2 * iz] + fr;
                    out64[2 * iz + 1] = out64[2 * iz + 1] + fq;
                }
            }
            if (ierr) break;
        }
    }
    ws_free(&w);
    return ierr;
}

/* ------------------------------------------------------------------------ */
/* graph: GENIEN -> GENID -> GENLM -> CONNECT -> GENCRS_QUICK -> CNMESH        */
/* (graph25_driver.f90:2-72)                                                 */
/* ------------------------------------------------------------------------ */
static int cmp_dbl_pair(const void *a, const void *b)
{
    const double *x = (const double *)a, *y = (const double *)b;
    if (x[0] < y[0]) return -1;
    if (x[0] > y[0]) return 1;
    if (x[1] < y[1]) return -1;
    if (x[1] > y[1]) return 1;
    return 0;
}
static int cmp_z_pair(const void *a, const void *b)
{
    const double *x = (const double *)a, *y = (const double *)b;
    if (x[1] < y[1]) return -1;
    if (x[1] > y[1]) return 1;
    return 0;
}
static int cmp_int(const void *a, const void *b)
{
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

/* IBSECT8 with JOB=1 (sort.f:1046-1105); vec is 1..n */
static int ibsect8(int n, double tol, double x, const double *vec)
{
    int r;
    if (fabs(x - vec[0]) < tol) return 1;
    if (fabs(x - vec[n - 1]) < tol) { r = n; goto back; }
    {
        int jl = 0, ju = n + 1, jm = 0;
        while (ju - jl > 1) {
            jm = (ju + jl) / 2;
            if ((vec[n - 1] >= vec[0]) == (x >= vec[jm - 1])) jl = jm;
            else ju = jm;
        }
        if (jl <= 0) return -1;
        if (fabs(vec[jl - 1] - x) < tol) r = jl;
        else if (jm >= 1 && jm <= n && fabs(vec[jm - 1] - x) < tol) r = jm;
        else if (ju >= 1 && ju <= n && fabs(vec[ju - 1] - x) < tol) r = ju;
        else return -1;
    }
back:
    for (int iloc = r; iloc >= 2; iloc--)
        if (fabs(vec[iloc - 1] - vec[iloc - 2]) > tol) return iloc;
    return r;
}

/* GENIEN (graph25.f:509-698): geometric de-duplication of element-edge
 * nodes (TOL 1e-8), sort by x then z within equal-x runs, edge nodes
 * numbered first, element-interior nodes after them in element order. */
static int genien(const orc_mesh *m, int nl, const double *pts, int *ien, int *nnp_out)
{
    const double TOL = 1e-8;
    int nelem = m->nelem, nen = nl * nl;
    long mnodes = (long)nelem * (2 * (nl - 1) + 2 * nl);
    double *xz = (double *)malloc(sizeof(double) * 2 * (mnodes + 1));
    long inodes = 0;
    /* kick out the repeats: linear scan over the distinct nodes found so far
     * (graph25.f:568-575); a spatial bucket index gives the same first-match
     * answer because distinct nodes are further than TOL apart. */
    double xmin = 1e300, xmax = -1e300, zmin = 1e300, zmax = -1e300;
    for (int p = 0; p < m->nnpg; p++) {
        if (m->xlocs[p] < xmin) xmin = m->xlocs[p];
        if (m->xlocs[p] > xmax) xmax = m->xlocs[p];
        if (m->zlocs[p] < zmin) zmin = m->zlocs[p];
        if (m->zlocs[p] > zmax) zmax = m->zlocs[p];
    }
    int nbx = 1024, nbz = 1024;
    double hx = (xmax - xmin) / nbx + 1e-6, hz = (zmax - zmin) / nbz + 1e-6;
    long *head = (long *)malloc(sizeof(long) * nbx * nbz);
    long *next = (long *)malloc(sizeof(long) * (mnodes + 1));
    for (long i = 0; i < (long)nbx * nbz; i++) head[i] = -1;
    for (int ielem = 0; ielem < nelem; ielem++) {
        const int *ieng = m->ieng + 4 * ielem;
        for (int ileta = 1; ileta <= nl; ileta++) {
            double eta = pts[ileta - 1];
            for (int ilxi = 1; ilxi <= nl; ilxi++) {
                if (!(ilxi == 1 || ilxi == nl || ileta == 1 || ileta == nl)) continue;
                double xi = pts[ilxi - 1], sf[4];
                csf2dnd(xi, eta, sf);
                double x = 0.0, z = 0.0;
                for (int ia = 0; ia < 4; ia++) {
                    x = x + sf[ia] * m->xlocs[ieng[ia] - 1];
                    z = z + sf[ia] * m->zlocs[ieng[ia] - 1];
                }
                int bx = (int)((x - xmin) / hx), bz = (int)((z - zmin) / hz);
                int found = 0;
                for (int dx = -1; dx <= 1 && !found; dx++)
                    for (int dz = -1; dz <= 1 && !found; dz++) {
                        int cx = bx + dx, cz = bz + dz;
                        if (cx < 0 || cz < 0 || cx >= nbx || cz >= nbz) continue;
                        for (long j = head[(long)cx * nbz + cz]; j >= 0; j = next[j])
                            if (fabs(xz[2 * j] - x) < TOL && fabs(xz[2 * j + 1] - z) < TOL) {
                                found = 1; break;
                            }
                    }
                if (found) continue;
                xz[2 * inodes] = x; xz[2 * inodes + 1] = z;
                if (bx < 0) bx = 0;
                if (bz < 0) bz = 0;
                if (bx >= nbx) bx = nbx - 1;
                if (bz >= nbz) bz = nbz - 1;
                next[inodes] = head[(long)bx * nbz + bz];
                head[(long)bx * nbz + bz] = inodes;
                inodes++;
            }
        }
    }
    free(head); free(next);
    long nnodes = inodes;
    /* heap sort on x (DHPSRT2); ties in x are resolved by the z sort below */
    qsort(xz, nnodes, 2 * sizeof(double), cmp_dbl_pair);
    /* shell sort z within runs of x equal to TOL (graph25.f:589-617) */
    long jbeg = 1;
    for (long in = 1; in <= nnodes; in++) {
        if (in + 1 == nnodes) {
            if (jbeg == nnodes) break;
            qsort(xz + 2 * (jbeg - 1), nnodes - jbeg + 1, 2 * sizeof(double), cmp_z_pair);
            break;
        }
        if (in + 1 > nnodes) break;
        if (fabs(xz[2 * in] - xz[2 * (in - 1)]) > TOL) {
            long jend = in;
            if (jend - jbeg + 1 > 1)
                qsort(xz + 2 * (jbeg - 1), jend - jbeg + 1, 2 * sizeof(double), cmp_z_pair);
            jbeg = jend + 1;
        }
    }
    long nnps = nnodes;
    double *xs = (double *)malloc(sizeof(double) * (nnps + 1));
    for (long i = 0; i < nnps; i++) xs[i] = xz[2 * i];
    xs[nnps] = 1.79769313486231571e308; /* HUGE */
    int iint = (int)nnps;
    int ierr = 0;
    for (int ielem = 0; ielem < nelem && !ierr; ielem++) {
        const int *ieng = m->ieng + 4 * ielem;
        for (int ileta = 1; ileta <= nl && !ierr; ileta++) {
            double eta = pts[ileta - 1];
            for (int ilxi = 1; ilxi <= nl; ilxi++) {
                int iae = (ileta - 1) * nl + ilxi;
                if (ilxi == 1 || ilxi == nl || ileta == 1 || ileta == nl) {
                    double xi = pts[ilxi - 1], sf[4];
                    csf2dnd(xi, eta, sf);
                    double x = 0.0, z = 0.0;
                    for (int ia = 0; ia < 4; ia++) {
                        x = x + sf[ia] * m->xlocs[ieng[ia] - 1];
                        z = z + sf[ia] * m->zlocs[ieng[ia] - 1];
                    }
                    int jb = ibsect8((int)nnps + 1, TOL, x, xs);
                    if (jb < 0 || fabs(xs[jb - 1] - x) > TOL) { ierr = 3; break; }
                    int fnd = 0;
                    for (long j = jb; j <= nnps; j++)
                        if (fabs(xz[2 * (j - 1)] - x) < TOL && fabs(xz[2 * (j - 1) + 1] - z) < TOL) {
                            ien[(size_t)ielem * nen + iae - 1] = (int)j; fnd = 1; break;
                        }
                    if (!fnd) { ierr = 4; break; }
                } else {
                    iint++;
                    ien[(size_t)ielem * nen + iae - 1] = iint;
                }
            }
        }
    }
    free(xs); free(xz);
    *nnp_out = iint;
    return ierr;
}

static int is_fixed(const char *c)
{
    return (c[0] == 'F' && (c[1] == 'L' || c[1] == 'B' || c[1] == 'R'));
}

/* GENID (graph25.f:315-505) */
static int genid(const orc_mesh *m, int nl, const double *pts, const int *ien, int nnp, int *id,
                 int *ndof_out)
{
    const double TOL = 1e-10;
    const int LNULL = -5;
    int nen = nl * nl;
    for (int i = 0; i < 3 * nnp; i++) id[i] = LNULL;
    for (int ielem = 0; ielem < m->nelem; ielem++) {
        if (m->cdomain[ielem] != 'A') continue;
        const int *ieng = m->ieng + 4 * ielem;
        int icheck = 0, iav[3] = {0, 0, 0}, ia1 = 0, ia2 = 0;
        for (int ia = 0; ia < 4; ia++) {
            int iloc = ieng[ia];
            if (is_fixed(m->cnnpg + 2 * (iloc - 1))) {
                icheck++;
                ia1 = iloc;
                iav[icheck - 1] = ia1;
                for (int ja = 0; ja < 4; ja++) {
                    int jloc = ieng[ja];
                    if (is_fixed(m->cnnpg + 2 * (jloc - 1)) && iloc != jloc) {
                        icheck++;
                        ia2 = jloc;
                        iav[icheck - 1] = jloc;
                        if (icheck == 3) goto l20;
                    }
                }
                goto l20;
            }
        }
    l20:
        if (icheck == 0) continue;
        {
            double v1[3] = {0, 0, 0};
            ia1 = iav[0];
            for (int loop = 1; loop <= 2; loop++) {
                if (icheck > 1) {
                    ia1 = iav[loop - 1];
                    ia2 = (loop < 3) ? iav[loop] : 0;
                    if (loop == 2 && icheck == 2) ia2 = 0;
                    if (ia2 == 0) break;
                    v1[0] = m->xlocs[ia2 - 1] - m->xlocs[ia1 - 1];
                    v1[1] = 0.0;
                    v1[2] = m->zlocs[ia2 - 1] - m->zlocs[ia1 - 1];
                } else {
                    if (loop == 2) break;
                }
                for (int ileta = 1; ileta <= nl; ileta++) {
                    double eta = pts[ileta - 1];
                    for (int ilxi = 1; ilxi <= nl; ilxi++) {
                        int iae = (ileta - 1) * nl + ilxi;
                        if (!(ilxi == 1 || ilxi == nl || ileta == 1 || ileta == nl)) continue;
                        int inp = ien[(size_t)ielem * nen + iae - 1];
                        double sf[4];
                        csf2dnd(pts[ilxi - 1], eta, sf);
                        double x = 0.0, z = 0.0;
                        for (int ia = 0; ia < 4; ia++) {
                            x = x + sf[ia] * m->xlocs[ieng[ia] - 1];
                            z = z + sf[ia] * m->zlocs[ieng[ia] - 1];
                        }
                        if (icheck == 1) {
                            if (fabs(x - m->xlocs[ia1 - 1]) < TOL && fabs(z - m->zlocs[ia1 - 1]) < TOL) {
                                id[3 * (inp - 1)] = 0; id[3 * (inp - 1) + 1] = 0; id[3 * (inp - 1) + 2] = 0;
                            }
                        } else {
                            double v2[3];
                            v2[0] = x - m->xlocs[ia1 - 1];
                            v2[1] = 0.0;
                            v2[2] = z - m->zlocs[ia1 - 1];
                            double det = v1[0] * v2[2] - v1[2] * v2[0];
                            if (fabs(det) < TOL) {
                                id[3 * (inp - 1)] = 0; id[3 * (inp - 1) + 1] = 0; id[3 * (inp - 1) + 2] = 0;
                            }
                        }
                    }
                }
            }
        }
    }
    int idof = 0;
    for (int ielem = 0; ielem < m->nelem; ielem++)
        for (int iae = 0; iae < nen; iae++) {
            int inp = ien[(size_t)ielem * nen + iae];
            for (int i = 0; i < 3; i++)
                if (id[3 * (inp - 1) + i] == LNULL) { idof++; id[3 * (inp - 1) + i] = idof; }
        }
    *ndof_out = idof;
    for (int i = 0; i < 3 * nnp; i++) if (id[i] == LNULL) return 1;
    return 0;
}

/* CONNECT (graph25.f:41-86) on a generic element->node table */
static int *connect(int nn, int nelem, int npe, const int *ien, int *ncon_out)
{
    int *cnt = (int *)calloc(nn, sizeof(int));
    for (int e = 0; e < nelem; e++)
        for (int a = 0; a < npe; a++) cnt[ien[(size_t)e * npe + a] - 1]++;
    int ncon = 0;
    for (int i = 0; i < nn; i++) if (cnt[i] > ncon) ncon = cnt[i]; /* ICMCON */
    int *mconn = (int *)calloc((size_t)nn * ncon, sizeof(int)); /* MCONN(NNP,NCON) col-major */
    for (int e = 0; e < nelem; e++)
        for (int a = 0; a < npe; a++) {
            int inp = ien[(size_t)e * npe + a];
            for (int ic = 0; ic < ncon; ic++)
                if (mconn[(inp - 1) + (size_t)nn * ic] == 0) { mconn[(inp - 1) + (size_t)nn * ic] = e + 1; break; }
        }
    free(cnt);
    *ncon_out = ncon;
    return mconn;
}

orc_graph *orc_graph_build(const orc_mesh *m, int *ierr)
{
    int nl = m->nord + 1, nen = nl * nl;
    double pts[32];
    orc_genpts(nl, pts);
    orc_graph *g = (orc_graph *)calloc(1, sizeof(orc_graph));
    g->nen = nen; g->nelem = m->nelem;
    g->ien = (int *)malloc(sizeof(int) * (size_t)nen * m->nelem);
    *ierr = genien(m, nl, pts, g->ien, &g->nnp);
    if (*ierr) return g;
    int *id = (int *)malloc(sizeof(int) * 3 * (size_t)g->nnp);
    *ierr = genid(m, nl, pts, g->ien, g->nnp, id, &g->ndof);
    if (*ierr) { free(id); *ierr += 10; return g; }
    /* GENLM (graph25.f:1-37) */
    g->lm = (int *)malloc(sizeof(int) * 3 * (size_t)nen * m->nelem);
    for (int e = 0; e < m->nelem; e++)
        for (int a = 0; a < nen; a++)
            for (int i = 0; i < 3; i++)
                g->lm[((size_t)e * nen + a) * 3 + i] = id[3 * (g->ien[(size_t)e * nen + a] - 1) + i];
    free(id);
    int ncon;
    int *mconn = connect(g->nnp, m->nelem, nen, g->ien, &ncon);
    g->ncon = ncon;
    /* GENCRS_QUICK (graph25.f:136-266) */
    int ndof = g->ndof;
    int nwork = 3 * ncon * nen + 1;
    int *jz = (int *)malloc(sizeof(int) * (nwork + 1));
    long long cap = (long long)ndof * 64 + 1024, izero = 0;
    int *jcw = (int *)malloc(sizeof(int) * cap);
    int *irw = (int *)malloc(sizeof(int) * (ndof + 2));
    int *perm = (int *)calloc(ndof + 1, sizeof(int));
    int ifound = 0;
    irw[0] = 1;
    for (int e = 0; e < m->nelem; e++)
        for (int a = 0; a < nen; a++) {
            int inp = g->ien[(size_t)e * nen + a];
            for (int i = 0; i < 3; i++) {
                int idof = g->lm[((size_t)e * nen + a) * 3 + i];
                if (idof <= 0 || perm[idof] != 0) continue;
                int jrr = 0;
                for (int ic = 0; ic < ncon; ic++) {
                    int je = mconn[(inp - 1) + (size_t)g->nnp * ic];
                    if (je == 0) break;
                    for (int b = 0; b < nen; b++)
                        for (int j = 0; j < 3; j++) {
                            int jdof = g->lm[((size_t)(je - 1) * nen + b) * 3 + j];
                            if (jdof > 0) jz[jrr++] = jdof;
                        }
                }
                qsort(jz, jrr, sizeof(int), cmp_int); /* ISHELL1 */
                jz[jrr] = 0;
                for (int k = 0; k < jrr; k++)
                    if (jz[k] != jz[k + 1]) {
                        if (izero >= cap) { cap *= 2; jcw = (int *)realloc(jcw, sizeof(int) * cap); }
                        jcw[izero++] = jz[k];
                    }
                ifound++;
                perm[idof] = ifound;
                irw[ifound] = (int)izero + 1;
            }
        }
    g->nzero = izero;
    g->irptr = (int *)malloc(sizeof(int) * (ndof + 1));
    g->jcptr = (int *)malloc(sizeof(int) * (izero > 0 ? izero : 1));
    long long iz = 0;
    g->irptr[0] = 1;
    for (int idof = 1; idof <= ndof; idof++) {
        int irow = perm[idof];
        for (int jz0 = irw[irow - 1]; jz0 <= irw[irow] - 1; jz0++) g->jcptr[iz++] = jcw[jz0 - 1];
        g->irptr[idof] = (int)iz + 1;
    }
    free(jz); free(jcw); free(irw); free(perm); free(mconn);
    /* CNMESH (bielak_utils.f:934-1025) */
    g->cnp = (char *)malloc(ndof);
    memset(g->cnp, ' ', ndof);
    for (int e = 0; e < m->nelem; e++)
        if (m->cdomain[e] == 'A')
            for (int k = 0; k < 3 * nen; k++) {
                int idof = g->lm[(size_t)e * 3 * nen + k];
                if (idof > 0) g->cnp[idof - 1] = 'A';
            }
    for (int e = 0; e < m->nelem; e++)
        if (m->cdomain[e] == 'E')
            for (int k = 0; k < 3 * nen; k++) {
                int idof = g->lm[(size_t)e * 3 * nen + k];
                if (idof > 0 && g->cnp[idof - 1] == ' ') g->cnp[idof - 1] = 'E';
            }
    for (int e = 0; e < m->nelem; e++)
        if (m->cdomain[e] == 'I')
            for (int k = 0; k < 3 * nen; k++) {
                int idof = g->lm[(size_t)e * 3 * nen + k];
                if (idof <= 0) continue;
                if (g->cnp[idof - 1] == ' ') g->cnp[idof - 1] = 'I';
                else if (g->cnp[idof - 1] == 'E') g->cnp[idof - 1] = 'B';
                else if (g->cnp[idof - 1] == 'A') *ierr = 21;
            }
    for (int i = 0; i < ndof; i++) if (g->cnp[i] == ' ') *ierr = 22;
    return g;
}

void orc_graph_info(const orc_graph *g, int *nnp, int *ndof, long long *nzero, int *ncon)
{
    *nnp = g->nnp; *ndof = g->ndof; *nzero = g->nzero; *ncon = g->ncon;
}

void orc_graph_copy(const orc_graph *g, int *ien, int *lm, int *irptr, int *jcptr, char *cnp)
{
    size_t nen = g->nen, ne = g->nelem;
    if (ien) memcpy(ien, g->ien, sizeof(int) * nen * ne);
    if (lm) memcpy(lm, g->lm, sizeof(int) * 3 * nen * ne);
    if (irptr) memcpy(irptr, g->irptr, sizeof(int) * (g->ndof + 1));
    if (jcptr) memcpy(jcptr, g->jcptr, sizeof(int) * g->nzero);
    if (cnp) memcpy(cnp, g->cnp, g->ndof);
}

void orc_graph_free(orc_graph *g)
{
    if (!g) return;
    free(g->ien); free(g->lm); free(g->irptr); free(g->jcptr); free(g->cnp); free(g);
}

/* ------------------------------------------------------------------------ */
/* Bielak effective force: ASMB_PEFF (asmble.f90:318-377), COMPLEX*8          */
/* ------------------------------------------------------------------------ */
void orc_peff(int ndof, const int *irptr, const int *jcptr, const char *cnp, const float *cdist,
              const float *ue, float *peff)
{
    for (int i = 0; i < 2 * ndof; i++) peff[i] = 0.0f;
    for (int idof = 1; idof <= ndof; idof++) {
        char c1 = cnp[idof - 1];
        if (c1 != 'B' && c1 != 'E') continue;
        for (int j = irptr[idof - 1]; j <= irptr[idof] - 1; j++) {
            int jdof = jcptr[j - 1];
            char c2 = cnp[jdof - 1];
            float ar = cdist[2 * (j - 1)], ai = cdist[2 * (j - 1) + 1];
            float ur = ue[2 * (jdof - 1)], ui = ue[2 * (jdof - 1) + 1];
            float pr = ar * ur - ai * ui, pi = ar * ui + ai * ur;
            if (c1 == 'B' && c2 == 'E') {
                peff[2 * (idof - 1)] = peff[2 * (idof - 1)] - pr;
                peff[2 * (idof - 1) + 1] = peff[2 * (idof - 1) + 1] - pi;
            } else if (c1 == 'E' && c2 == 'B') {
                peff[2 * (idof - 1)] = peff[2 * (idof - 1)] + pr;
                peff[2 * (idof - 1) + 1] = peff[2 * (idof - 1) + 1] + pi;
            }
        }
    }
}

/* ADDBLK (bielak_utils.f:1116-1125): the Bielak background field is added
 * back into the total solution on the exterior DOFs, SOL(i) = SOL(i) + U0(i)
 * for CNP(i) = 'E', in COMPLEX*8 (callers funcgradh.f90:248,
 * srcrec.f90:694). */
void orc_addblk(int ndof, const char *cnp, const float *u0, float *sol)
{
    for (int idof = 1; idof <= ndof; idof++) {
        if (cnp[idof - 1] != 'E') continue;
        sol[2 * (idof - 1)] = sol[2 * (idof - 1)] + u0[2 * (idof - 1)];
        sol[2 * (idof - 1) + 1] = sol[2 * (idof - 1) + 1] + u0[2 * (idof - 1) + 1];
    }
}

/* VERIFY_STEVE (asmble.f90:381-433), the Bielak identity check: on every
 * exterior ('E') row, BUFF1 = sum over 'E' and 'B' columns of S_ij U0_j and
 * BUFF2 = the same sum over the solved total field SOL (after ADDBLK), in
 * COMPLEX*8 and the row's column order; returns DIF1 = max |BUFF1 - BUFF2|
 * (the reference prints it).  With P_eff from ASMB_PEFF the two agree up to
 * the solve's residual on the 'E' rows; buff1 / buff2 (nullable, COMPLEX*8
 * [NDOF], zero off the 'E' rows) return the sums. */
float orc_verify_steve(int ndof, const int *irptr, const int *jcptr, const char *cnp,
                       const float *cdist, const float *u0, const float *sol, float *buff1,
                       float *buff2)
{
    float dif1 = 0.0f;
    for (int idof = 1; idof <= ndof; idof++) {
        float b1r = 0.0f, b1i = 0.0f, b2r = 0.0f, b2i = 0.0f;
        if (cnp[idof - 1] == 'E') {
            for (int j = irptr[idof - 1]; j <= irptr[idof] - 1; j++) {
                int jdof = jcptr[j - 1];
                char c2 = cnp[jdof - 1];
                if (c2 != 'B' && c2 != 'E') continue;
                float ar = cdist[2 * (j - 1)], ai = cdist[2 * (j - 1) + 1];
                float ur = u0[2 * (jdof - 1)], ui = u0[2 * (jdof - 1) + 1];
                float sr = sol[2 * (jdof - 1)], si = sol[2 * (jdof - 1) + 1];
                b1r = b1r + (ar * ur - ai * ui);
                b1i = b1i + (ar * ui + ai * ur);
                b2r = b2r + (ar * sr - ai * si);
                b2i = b2i + (ar * si + ai * sr);
            }
        }
        if (buff1) { buff1[2 * (idof - 1)] = b1r; buff1[2 * (idof - 1) + 1] = b1i; }
        if (buff2) { buff2[2 * (idof - 1)] = b2r; buff2[2 * (idof - 1) + 1] = b2i; }
        float dr = b1r - b2r, di = b1i - b2i;
        float d = sqrtf(dr * dr + di * di);
        if (d > dif1) dif1 = d;
    }
    return dif1;
}

/* ------------------------------------------------------------------------ */
/* exact adjoint gradient in anchor-node lambda, mu, rho                      */
/* g[m*nnpg + p] += sum_s Re( lam_s^H (dA/dm_p) u_s ) over non-PML elements.  */
/* KM25ISOQ is linear in the quadrature-point lambda, mu, rho, so dA_e/dm_p   */
/* is KM25ISOQ with that field replaced by the bilinear anchor shape function */
/* SF_p (cjac.f:98-108) and the other two fields set to zero.                 */
/* u, lam: complex128 [nsrc][ndof] interleaved.                               */
/* ------------------------------------------------------------------------ */
int orc_grad_exact(const orc_mesh *m, const int *lm, int ndof, double freq, double py, int nsrc,
                   const double *u, const double *lam, double *g)
{
    const double TWOPI = 6.2831853071795862;
    double omega = TWOPI * freq;
    orc_ws w;
    ws_init(&w, m->nord);
    int nen = w.nen, nee = w.nee, nq = w.nq, nint = w.nint;
    const double *wts = w.xigll + nint;
    double *fld[3], *zero = (double *)calloc(nq, sizeof(double)), *sfa = (double *)malloc(sizeof(double) * nq);
    zc *ue = (zc *)malloc(sizeof(zc) * nee), *le = (zc *)malloc(sizeof(zc) * nee);
    int ierr = 0;
    for (int e = 0; e < m->nelem && !ierr; e++) {
        if (m->cdomain[e] == 'A') continue;
        ierr = cjmk_tvi(m, e, nen, nint, w.xigll, w.shl, w.det, w.rho, w.vlam, w.vmu, w.shg);
        if (ierr) break;
        const int *lme = lm + (size_t)3 * nen * e;
        for (int a = 0; a < 4; a++) {
            for (int intx = 0; intx < nint; intx++)
                for (int intz = 0; intz < nint; intz++) {
                    double sf[4], dsf[8];
                    csf2d(w.xigll[intx], w.xigll[intz], sf, dsf);
                    sfa[intx + nint * intz] = sf[a];
                }
            int p = m->ieng[4 * e + a] - 1;
            for (int par = 0; par < 3; par++) {
                fld[0] = zero; fld[1] = zero; fld[2] = zero;
                fld[par] = sfa;
                km25isoq(nen, nint, omega, py, wts, fld[0], fld[1], fld[2], w.det, w.shg, w.me, w.ke);
                double acc = 0.0;
                for (int s = 0; s < nsrc; s++) {
                    for (int k = 0; k < nee; k++) {
                        int d = lme[k];
                        if (d > 0) {
                            ue[k] = zmk(u[2 * ((size_t)s * ndof + d - 1)], u[2 * ((size_t)s * ndof + d - 1) + 1]);
                            le[k] = zmk(lam[2 * ((size_t)s * ndof + d - 1)], lam[2 * ((size_t)s * ndof + d - 1) + 1]);
                        } else {
                            ue[k] = zmk(0.0, 0.0); le[k] = zmk(0.0, 0.0);
                        }
                    }
                    for (int i = 0; i < nee; i++) {
                        zc row = zmk(0.0, 0.0);
                        for (int j = 0; j < nee; j++) {
                            zc aij = zadd(zmk(w.me[i + nee * j], 0.0), w.ke[i + nee * j]);
                            row = zadd(row, zmul(aij, ue[j]));
                        }
                        /* Re(conj(lam_i) * row) */
                        acc = acc + (le[i].re * row.re + le[i].im * row.im);
                    }
                }
                g[(size_t)par * m->nnpg + p] += acc;
            }
        }
    }
    free(zero); free(sfa); free(ue); free(le);
    ws_free(&w);
    return ierr;
}

/* ------------------------------------------------------------------------ */
/* reference-compatible gradient: GENGMASK / ELEM_WTS / GRADPTRS /            */
/* CFMAT_DIST(VFORCE25, DJACAB, DKM_VPVS) / ADJFLAM_DIST                      */
/* ------------------------------------------------------------------------ */
/* GENGMASK (gengmask.f90:1-262) with no mask file, LINREC=.TRUE.,
 * LKBDRY=.TRUE., one partition.  mconn: MCONN(NNPG,NCON) over anchors. */
int orc_gengmask(const orc_mesh *m, const int *lm, int nord, int *maskg, int *mconn_out,
                 int *ncon_out)
{
    int ncon;
    int *mconn = connect(m->nnpg, m->nelem, 4, m->ieng, &ncon);
    int nl = nord + 1, nen = nl * nl;
    int inpinv = 0;
    for (int p = 0; p < m->nnpg; p++) {
        int keep = 1, e = mconn[p];
        if (e > 0 && m->cdomain[e - 1] != 'I') keep = 0;
        const char *c = m->cnnpg + 2 * p;
        if (keep && ((c[0] == 'I' && c[1] == 'I') || (c[0] == 'B' && c[1] == 'I') ||
                     (c[0] == 'F' && c[1] == 'S')))
            maskg[p] = ++inpinv;
        else
            maskg[p] = 0;
    }
    int lshift = 0;
    for (int e = 0; e < m->nelem; e++)
        for (int ia = 0; ia < 4; ia++) {
            int inpg = m->ieng[4 * e + ia];
            if (maskg[inpg - 1] > 0) {
                /* IA2IAE: anchor ia -> corner element node (1, NLXI, NEN, NEN-NLXI+1) */
                int iae = (ia == 0) ? 1 : (ia == 1) ? nl : (ia == 2) ? nen : nen - nl + 1;
                for (int i = 0; i < 3; i++)
                    if (lm[((size_t)e * nen + iae - 1) * 3 + i] <= 0) { maskg[inpg - 1] = 0; lshift = 1; break; }
            }
        }
    if (lshift) {
        inpinv = 0;
        for (int p = 0; p < m->nnpg; p++) if (maskg[p] > 0) maskg[p] = ++inpinv;
    }
    if (mconn_out) memcpy(mconn_out, mconn, sizeof(int) * (size_t)m->nnpg * ncon);
    *ncon_out = ncon;
    free(mconn);
    return inpinv;
}

int orc_ncon_anchor(const orc_mesh *m)
{
    int ncon;
    int *mc = connect(m->nnpg, m->nelem, 4, m->ieng, &ncon);
    free(mc);
    return ncon;
}

/* ELEM_WTS (gengmask.f90:758-841) */
void orc_elem_wts(const orc_mesh *m, const int *maskg, const int *mconn, int ncon, double *wts)
{
    char *linit = (char *)calloc(m->nelem, 1);
    double wtmax = 0.0;
    for (int e = 0; e < m->nelem; e++) wts[e] = 0.0;
    for (int p = 0; p < m->nnpg; p++) {
        if (maskg[p] <= 0) continue;
        for (int ic = 0; ic < ncon; ic++) {
            int e = mconn[p + (size_t)m->nnpg * ic];
            if (e <= 0) break;
            if (linit[e - 1]) continue;
            double rloc = 0.0;
            for (int ia1 = 1; ia1 <= 4; ia1++) {
                int j1 = m->ieng[4 * (e - 1) + ia1 - 1];
                int ia2 = (ia1 + 1) % 5;
                if (ia2 == 0) ia2 = 1;
                int j2 = m->ieng[4 * (e - 1) + ia2 - 1];
                double x1 = m->xlocs[j1 - 1], x2 = m->xlocs[j2 - 1];
                double z1 = m->zlocs[j1 - 1], z2 = m->zlocs[j2 - 1];
                rloc = rloc + x1 * z2 - x2 * z1;
            }
            if (rloc <= 0.0) rloc = -rloc;
            rloc = rloc * 0.5;
            wts[e - 1] = rloc;
            linit[e - 1] = 1;
            if (rloc > wtmax) wtmax = rloc;
        }
    }
    for (int e = 0; e < m->nelem; e++) if (wts[e] > 0.0) wts[e] = wtmax / wts[e];
    free(linit);
}

/* GRADPTRS (gengmask.f90:962-1118), one process, NVINV=1.
 * jcsc: [nnpinv+1], icsc: [nz] (pass NULL to count). Returns nz. */
long long orc_gradptrs(const orc_mesh *m, const int *lm, int nord, const int *maskg,
                       const int *mconn, int ncon, int *jcsc, int *icsc)
{
    int nl = nord + 1, nen = nl * nl;
    int *irow = (int *)malloc(sizeof(int) * (ncon * 3 * nen + 1));
    long long inzfl = 0;
    int inpgl = 1;
    if (jcsc) jcsc[0] = 1;
    for (int p = 0; p < m->nnpg; p++) {
        if (maskg[p] <= 0) continue;
        int n = 0;
        for (int ic = 0; ic < ncon; ic++) {
            int e = mconn[p + (size_t)m->nnpg * ic];
            if (e <= 0) break;
            for (int k = 0; k < 3 * nen; k++) {
                int d = lm[(size_t)(e - 1) * 3 * nen + k];
                if (d > 0) irow[n++] = d;
            }
        }
        qsort(irow, n, sizeof(int), cmp_int);
        irow[n] = 0;
        for (int k = 0; k < n; k++)
            if (irow[k + 1] != irow[k]) {
                if (icsc) icsc[inzfl] = irow[k];
                inzfl++;
            }
        if (jcsc) jcsc[inpgl] = (int)inzfl + 1;
        inpgl++;
    }
    free(irow);
    return inzfl;
}

/* DJACAB (djac.f:1-139) */
static int djacab(const orc_mesh *m, int ielem, int inpg, int nen, int nint, const double *xigll,
                  const double *shl, double *det, double *dab1, double *dab2, double *shg)
{
    const double EPS = 2.22e-16;
    const int *ieng = m->ieng + 4 * ielem;
    int nnpg = m->nnpg;
    for (int intx = 0; intx < nint; intx++) {
        double xi = xigll[intx];
        for (int intz = 0; intz < nint; intz++) {
            double eta = xigll[intz];
            double sf[4], dsf[8];
            if (csf2d(xi, eta, sf, dsf)) return 1;
            double x = 0.0, z = 0.0, dxdxi = 0.0, dxdeta = 0.0, dzdxi = 0.0, dzdeta = 0.0;
            int q = intx + nint * intz;
            dab1[q] = 0.0; dab2[q] = 0.0;
            for (int ia = 0; ia < 4; ia++) {
                int iloc = ieng[ia];
                double alpha, beta;
                if (iloc == inpg) {
                    alpha = sqrt((m->ecoeff[iloc - 1] + 2.0 * m->ecoeff[iloc - 1 + nnpg]) / m->dens[iloc - 1]);
                    beta = sqrt(m->ecoeff[iloc - 1 + nnpg] / m->dens[iloc - 1]);
                } else {
                    alpha = 0.0; beta = 0.0;
                }
                dab1[q] = dab1[q] + 2.0 * alpha * sf[ia];
                dab2[q] = dab2[q] + 2.0 * beta * sf[ia];
                x = x + sf[ia] * m->xlocs[iloc - 1];
                z = z + sf[ia] * m->zlocs[iloc - 1];
                dxdxi = dxdxi + dsf[0 + 2 * ia] * m->xlocs[iloc - 1];
                dxdeta = dxdeta + dsf[1 + 2 * ia] * m->xlocs[iloc - 1];
                dzdxi = dzdxi + dsf[0 + 2 * ia] * m->zlocs[iloc - 1];
                dzdeta = dzdeta + dsf[1 + 2 * ia] * m->zlocs[iloc - 1];
            }
            double rjac = dxdxi * dzdeta - dxdeta * dzdxi;
            det[q] = rjac;
            if (fabs(rjac) <= EPS || rjac < 0.0) return 1;
            fill_shg(nen, nint, intx, intz, shl, dxdxi, dxdeta, dzdxi, dzdeta, rjac, shg);
        }
    }
    return 0;
}

/* DKM_VPVS (dstiff25.f:498-662) */
static void dkm_vpvs(int nen, int nint, double omega, double py, const double *wts,
                     const double *dvp, const double *dvs, const double *det, const double *shg,
                     double *dme, zc *dke)
{
    int nee = nen * NDIM;
    for (int i = 0; i < nee * nee; i++) { dme[i] = 0.0; dke[i] = zmk(0.0, 0.0); }
    double wpy = omega * py, py2 = ipow(py, 2), w2 = ipow(omega, 2);
    for (int intx = 0; intx < nint; intx++)
        for (int intz = 0; intz < nint; intz++) {
            int q = intx + nint * intz;
            double weight = wts[intx] * wts[intz] * det[q];
            double drvp = dvp[q] * weight, drvs = dvs[q] * weight;
            double rm1 = w2 * py2 * drvs, rm2 = w2 * py2 * drvp, rm3 = rm1;
            (void)rm3;
            for (int ibe = 0; ibe < nen; ibe++) {
                size_t bb = 3 * ((size_t)ibe + (size_t)nen * q);
                double phib = shg[bb + 2], phibx = shg[bb + 0], phibz = shg[bb + 1];
                double rm11t1 = rm1 * phib, rm22t1 = rm2 * phib;
                double rk11t1 = drvp * phibx, rk11t2 = drvs * phibz;
                double rk13t1 = drvp * phibz, rk13t2 = drvs * phibx, rk13t3 = -2.0 * drvs * phibz;
                double rk22t1 = drvs * phibx, rk22t2 = drvs * phibz;
                double rk31t1 = drvp * phibx, rk31t2 = drvs * phibz, rk31t3 = -2.0 * drvs * phibx;
                double rk33t1 = drvp * phibz, rk33t2 = drvs * phibx;
                double rk12t1 = wpy * drvp * phib, rk12t2 = -2.0 * wpy * drvs * phib, rk12t3 = -wpy * drvs * phibx;
                double rk21t1 = wpy * drvp * phibx, rk21t2 = -2.0 * wpy * drvs * phibx, rk21t3 = -wpy * drvs * phib;
                double rk23t1 = wpy * drvp * phibz, rk23t2 = -2.0 * wpy * drvs * phibz, rk23t3 = -wpy * drvs * phib;
                double rk32t1 = wpy * drvp * phib, rk32t2 = -2.0 * wpy * drvs * phib, rk32t3 = -wpy * drvs * phibz;
                for (int iae = 0; iae < nen; iae++) {
                    size_t ab = 3 * ((size_t)iae + (size_t)nen * q);
                    double phia = shg[ab + 2], phiax = shg[ab + 0], phiaz = shg[ab + 1];
                    double rme11 = rm11t1 * phia, rme22 = rm22t1 * phia, rme33 = rme11;
                    double rke11 = rk11t1 * phiax + rk11t2 * phiaz;
                    double rke13 = rk13t1 * phiax + rk13t2 * phiaz + rk13t3 * phiax;
                    double rke22 = rk22t1 * phiax + rk22t2 * phiaz;
                    double rke31 = rk31t1 * phiaz + rk31t2 * phiax + rk31t3 * phiaz;
                    double rke33 = rk33t1 * phiaz + rk33t2 * phiax;
                    double rke12 = rk12t1 * phiax + rk12t2 * phiax + rk12t3 * phia;
                    double rke21 = rk21t1 * phia + rk21t2 * phia + rk21t3 * phiax;
                    double rke23 = rk23t1 * phia + rk23t2 * phia + rk23t3 * phiaz;
                    double rke32 = rk32t1 * phiaz + rk32t2 * phiaz + rk32t3 * phia;
                    int ipe = NDIM * iae, iqe = NDIM * ibe;
#define DME(i, j) dme[(i) + nee * (j)]
#define DKE(i, j) dke[(i) + nee * (j)]
                    DME(ipe, iqe) = DME(ipe, iqe) + rme11;
                    DME(ipe + 1, iqe + 1) = DME(ipe + 1, iqe + 1) + rme22;
                    DME(ipe + 2, iqe + 2) = DME(ipe + 2, iqe + 2) + rme33;
                    DKE(ipe, iqe) = zadd(DKE(ipe, iqe), zmk(rke11, 0.0));
                    DKE(ipe + 1, iqe + 1) = zadd(DKE(ipe + 1, iqe + 1), zmk(rke22, 0.0));
                    DKE(ipe + 2, iqe + 2) = zadd(DKE(ipe + 2, iqe + 2), zmk(rke33, 0.0));
                    DKE(ipe, iqe + 2) = zadd(DKE(ipe, iqe + 2), zmk(rke13, 0.0));
                    DKE(ipe + 2, iqe) = zadd(DKE(ipe + 2, iqe), zmk(rke31, 0.0));
                    DKE(ipe, iqe + 1) = zsub(DKE(ipe, iqe + 1), zmk(rke12, 0.0));
                    DKE(ipe + 1, iqe) = zadd(DKE(ipe + 1, iqe), zmk(rke21, 0.0));
                    DKE(ipe + 1, iqe + 2) = zadd(DKE(ipe + 1, iqe + 2), zmk(rke23, 0.0));
                    DKE(ipe + 2, iqe + 1) = zsub(DKE(ipe + 2, iqe + 1), zmk(rke32, 0.0));
                }
            }
        }
}

/* DABMKISOB25 (dstiff25.f:1-203): derivatives of the density-normalised
 * element operator with respect to the anchor's alpha (LISP) and beta (LISS)
 * with DAB from DJACAB (2 alpha N_p, 2 beta N_p).  The reference resets
 * DMDA(IPE,IQE) and DMDA(IPE+2,IQE+2) to zero and copies DMDB(IPE,IQE) into
 * DMDB(IPE+2,IQE+2) at every point (dstiff25.f:133-143); kept. */
static void dabmkisob25(int nen, int nint, int lisp, int liss, double omega, double py,
                        const double *wts, const double *det, const double *dab1,
                        const double *dab2, const double *shg, double *dmda, double *dmdb,
                        zc *dkda, zc *dkdb)
{
    int nee = nen * NDIM;
    for (int i = 0; i < nee * nee; i++) {
        dmda[i] = 0.0; dmdb[i] = 0.0; dkda[i] = zmk(0.0, 0.0); dkdb[i] = zmk(0.0, 0.0);
    }
    double wpy = omega * py, wpy2 = ipow(omega * py, 2);
    for (int intx = 0; intx < nint; intx++)
        for (int intz = 0; intz < nint; intz++) {
            int q = intx + nint * intz;
            double weight = wts[intx] * wts[intz] * det[q];
            double dalpha = dab1[q] * weight, dbeta = dab2[q] * weight;
            double dmassda = wpy2 * dalpha, dmassdb = wpy2 * dbeta;
            for (int ibe = 0; ibe < nen; ibe++) {
                size_t bb = 3 * ((size_t)ibe + (size_t)nen * q);
                double phib = shg[bb + 2], phibx = shg[bb + 0], phibz = shg[bb + 1];
                double dmdat1 = 0.0, dk11da = 0.0, dk13da = 0.0, dk31da = 0.0, dk33da = 0.0;
                double dk12da = 0.0, dk21da = 0.0, dk23da = 0.0, dk32da = 0.0;
                double dmdbt1 = 0.0, dk11dbt1 = 0.0, dk13dbt1 = 0.0, dk13dbt2 = 0.0;
                double dk22dbt1 = 0.0, dk22dbt2 = 0.0, dk31dbt1 = 0.0, dk31dbt2 = 0.0;
                double dk33dbt1 = 0.0, dk12dbt1 = 0.0, dk12dbt2 = 0.0, dk21dbt1 = 0.0;
                double dk21dbt2 = 0.0, dk23dbt1 = 0.0, dk23dbt2 = 0.0, dk32dbt1 = 0.0;
                double dk32dbt2 = 0.0;
                if (lisp) {
                    dmdat1 = dmassda * phib;
                    dk11da = dalpha * phibx;
                    dk13da = dalpha * phibz;
                    dk31da = dalpha * phibx;
                    dk33da = dalpha * phibz;
                    dk12da = wpy * dalpha * phib;
                    dk21da = wpy * dalpha * phibx;
                    dk23da = wpy * dalpha * phibz;
                    dk32da = wpy * dalpha * phib;
                }
                if (liss) {
                    dmdbt1 = dmassdb * phib;
                    dk11dbt1 = dbeta * phibz;
                    dk13dbt1 = dbeta * phibx;
                    dk13dbt2 = -(2.0 * dbeta * phibz);
                    dk22dbt1 = dbeta * phibx;
                    dk22dbt2 = dbeta * phibz;
                    dk31dbt1 = dbeta * phibz;
                    dk31dbt2 = -(2.0 * dbeta * phibx);
                    dk33dbt1 = dbeta * phibx;
                    dk12dbt1 = 2.0 * wpy * dbeta * phib;
                    dk12dbt2 = wpy * dbeta * phibx;
                    dk21dbt1 = 2.0 * wpy * dbeta * phibx;
                    dk21dbt2 = wpy * dbeta * phib;
                    dk23dbt1 = 2.0 * wpy * dbeta * phibz;
                    dk23dbt2 = wpy * dbeta * phib;
                    dk32dbt1 = 2.0 * wpy * dbeta * phib;
                    dk32dbt2 = wpy * dbeta * phibz;
                }
                for (int iae = 0; iae < nen; iae++) {
                    size_t ab = 3 * ((size_t)iae + (size_t)nen * q);
                    double phia = shg[ab + 2], phiax = shg[ab + 0], phiaz = shg[ab + 1];
                    int ipe = NDIM * iae, iqe = NDIM * ibe;
#define DMDA(i, j) dmda[(i) + nee * (j)]
#define DMDB(i, j) dmdb[(i) + nee * (j)]
#define DKDA(i, j) dkda[(i) + nee * (j)]
#define DKDB(i, j) dkdb[(i) + nee * (j)]
                    if (lisp) {
                        DMDA(ipe, iqe) = 0.0;
                        DMDA(ipe + 1, iqe + 1) = DMDA(ipe + 1, iqe + 1) + dmdat1 * phia;
                        DMDA(ipe + 2, iqe + 2) = 0.0;
                    }
                    if (liss) {
                        DMDB(ipe, iqe) = DMDB(ipe, iqe) + dmdbt1 * phia;
                        DMDB(ipe + 1, iqe + 1) = 0.0;
                        DMDB(ipe + 2, iqe + 2) = DMDB(ipe, iqe);
                    }
                    if (lisp) {
                        zc dke11 = zmk(phiax * dk11da, 0.0), dke13 = zmk(phiax * dk13da, 0.0);
                        zc dke22 = zmk(0.0, 0.0);
                        zc dke31 = zmk(phiaz * dk31da, 0.0), dke33 = zmk(phiaz * dk33da, 0.0);
                        zc dke12 = zmk(0.0, phiax * dk12da), dke21 = zmk(0.0, phia * dk21da);
                        zc dke23 = zmk(0.0, phia * dk23da), dke32 = zmk(0.0, phiaz * dk32da);
                        DKDA(ipe, iqe) = zadd(DKDA(ipe, iqe), dke11);
                        DKDA(ipe, iqe + 1) = zsub(DKDA(ipe, iqe + 1), dke12);
                        DKDA(ipe, iqe + 2) = zadd(DKDA(ipe, iqe + 2), dke13);
                        DKDA(ipe + 1, iqe) = zadd(DKDA(ipe + 1, iqe), dke21);
                        DKDA(ipe + 1, iqe + 1) = zadd(DKDA(ipe + 1, iqe + 1), dke22);
                        DKDA(ipe + 1, iqe + 2) = zadd(DKDA(ipe + 1, iqe + 2), dke23);
                        DKDA(ipe + 2, iqe) = zadd(DKDA(ipe + 2, iqe), dke31);
                        DKDA(ipe + 2, iqe + 1) = zsub(DKDA(ipe + 2, iqe + 1), dke32);
                        DKDA(ipe + 2, iqe + 2) = zadd(DKDA(ipe + 2, iqe + 2), dke33);
                    }
                    if (liss) {
                        zc dke11 = zmk(phiaz * dk11dbt1, 0.0);
                        zc dke13 = zmk(phiaz * dk13dbt1 + phiax * dk13dbt2, 0.0);
                        zc dke22 = zmk(phiax * dk22dbt1 + phiaz * dk22dbt2, 0.0);
                        zc dke31 = zmk(phiax * dk31dbt1 + phiaz * dk31dbt2, 0.0);
                        zc dke33 = zmk(phiax * dk33dbt1, 0.0);
                        zc dke12 = zmk(0.0, phiax * dk12dbt1 + phia * dk12dbt2);
                        zc dke21 = zmk(0.0, phia * dk21dbt1 + phiax * dk21dbt2);
                        zc dke23 = zmk(0.0, phia * dk23dbt1 + phiaz * dk23dbt2);
                        zc dke32 = zmk(0.0, phiaz * dk32dbt1 + phia * dk32dbt2);
                        DKDB(ipe, iqe) = zadd(DKDB(ipe, iqe), dke11);
                        DKDB(ipe, iqe + 1) = zadd(DKDB(ipe, iqe + 1), dke12);
                        DKDB(ipe, iqe + 2) = zadd(DKDB(ipe, iqe + 2), dke13);
                        DKDB(ipe + 1, iqe) = zsub(DKDB(ipe + 1, iqe), dke21);
                        DKDB(ipe + 1, iqe + 1) = zadd(DKDB(ipe + 1, iqe + 1), dke22);
                        DKDB(ipe + 1, iqe + 2) = zsub(DKDB(ipe + 1, iqe + 2), dke23);
                        DKDB(ipe + 2, iqe) = zadd(DKDB(ipe + 2, iqe), dke31);
                        DKDB(ipe + 2, iqe + 1) = zadd(DKDB(ipe + 2, iqe + 1), dke32);
                        DKDB(ipe + 2, iqe + 2) = zadd(DKDB(ipe + 2, iqe + 2), dke33);
                    }
                }
            }
        }
}

/* exported: DABMKISOB25 matrices of element ielem for anchor inpg (1-based) */
int orc_dabm_element(const orc_mesh *m, int ielem, int inpg, double freq, double py,
                     double *dmda, double *dkda, double *dmdb, double *dkdb)
{
    const double TWOPI = 6.2831853071795862;
    orc_ws w;
    ws_init(&w, m->nord);
    double *dab1 = (double *)malloc(sizeof(double) * w.nq), *dab2 = (double *)malloc(sizeof(double) * w.nq);
    int ierr = djacab(m, ielem, inpg, w.nen, w.nint, w.xigll, w.shl, w.det, dab1, dab2, w.shg);
    if (!ierr)
        dabmkisob25(w.nen, w.nint, 1, 1, TWOPI * freq, py, w.xigll + w.nint, w.det, dab1, dab2,
                    w.shg, dmda, dmdb, (zc *)dkda, (zc *)dkdb);
    free(dab1); free(dab2);
    ws_free(&w);
    return ierr;
}

typedef struct { float re, im; } cc;
static inline cc cmk(float a, float b) { cc z; z.re = a; z.im = b; return z; }
static inline cc cmulf(cc a, cc b) { return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }

/*
 * CFMAT_DIST (hessloc.f90:1-133) -> VFORCE25 (vforce25.f:1-369), one
 * process, NVINV=1 ('PP' -> lisp=1, 'SS' -> lisp=0).  wave: COMPLEX*8
 * [ndof]; fmat: COMPLEX*8 [nz].  Inversion anchors are visited in MASKG
 * order.  VFORCE25 nulls the force column inside its loop over connected
 * elements (vforce25.f:274-280), so only the last connected element's
 * contribution survives; `accumulate`=1 keeps every element instead.
 */
int orc_cfmat_dist(const orc_mesh *m, const int *lm, int ndof, const int *maskg,
                   const int *mconn, int ncon, const double *elem_wts, const int *jcsc,
                   const int *icsc, int lisp, double vpvs, double freq, double py,
                   const float *wave, float *fmat, int accumulate)
{
    const double TWOPI = 6.2831853071795862;
    double omega = TWOPI * freq, vpvs2 = vpvs * vpvs;
    orc_ws w;
    ws_init(&w, m->nord);
    int nen = w.nen, nee = w.nee, nq = w.nq, nint = w.nint;
    const double *wts = w.xigll + nint;
    double *dab1 = (double *)malloc(sizeof(double) * nq), *dab2 = (double *)malloc(sizeof(double) * nq);
    double *dvp = (double *)malloc(sizeof(double) * nq), *dvs = (double *)malloc(sizeof(double) * nq);
    int ierr = 0, inpgl = 0;
    (void)ndof;
    for (int p = 0; p < m->nnpg && !ierr; p++) {
        if (maskg[p] <= 0) continue;
        inpgl++;
        int i1 = jcsc[inpgl - 1], i2 = jcsc[inpgl] - 1, nnzrow = i2 - i1 + 1;
        float *forcev = fmat + 2 * (size_t)(i1 - 1);
        for (int k = 0; k < 2 * nnzrow; k++) forcev[k] = 0.0f;
        for (int ic = 0; ic < ncon; ic++) {
            int e = mconn[p + (size_t)m->nnpg * ic];
            if (e <= 0) break;
            ierr = djacab(m, e - 1, p + 1, nen, nint, w.xigll, w.shl, w.det, dab1, dab2, w.shg);
            if (ierr) break;
            for (int q = 0; q < nq; q++) {
                if (lisp) { dvp[q] = dab1[q]; dvs[q] = dab1[q] / vpvs2; }
                else { dvp[q] = dab2[q] * vpvs2; dvs[q] = dab2[q]; }
            }
            dkm_vpvs(nen, nint, omega, py, wts, dvp, dvs, w.det, w.shg, w.me, w.ke);
            if (!accumulate) for (int k = 0; k < 2 * nnzrow; k++) forcev[k] = 0.0f;
            cc cwght = cmk((float)elem_wts[e - 1], 0.0f);
            const int *lme = lm + (size_t)3 * nen * (e - 1);
            for (int ipe = 0; ipe < nee; ipe++) {
                int idof = lme[ipe];
                if (idof <= 0) continue;
                int inz = ibsect(nnzrow, idof, icsc + (i1 - 1));
                if (inz <= 0 || inz > nnzrow) { ierr = 3; break; }
                for (int iqe = 0; iqe < nee; iqe++) {
                    int jdof = lme[iqe];
                    if (jdof <= 0) continue;
                    double ar = w.me[ipe + nee * iqe] + w.ke[ipe + nee * iqe].re;
                    double ai = 0.0 + w.ke[ipe + nee * iqe].im;
                    cc carg = cmk((float)ar, (float)ai);
                    cc wv = cmk(wave[2 * (jdof - 1)], wave[2 * (jdof - 1) + 1]);
                    cc t = cmulf(cmulf(carg, wv), cwght);
                    forcev[2 * (inz - 1)] = forcev[2 * (inz - 1)] + t.re;
                    forcev[2 * (inz - 1) + 1] = forcev[2 * (inz - 1) + 1] + t.im;
                }
            }
            if (ierr) break;
        }
    }
    free(dab1); free(dab2); free(dvp); free(dvs);
    ws_free(&w);
    return ierr;
}

/*
 * VFORCE25_2 (vforce25.f:373-607) for every inversion anchor (MASKG order):
 * F_p(row, ivinv) += CMPLX(DCMPLX(DMD*,0) + DKD*)(row, col) * WAVE(col) over
 * the connected elements in MCONN order, COMPLEX*8 arithmetic, no element
 * weights and no reset between elements.  Rows are the CSC pattern of
 * GRADPTRS.  fmat: COMPLEX*8 [nvinv][nz], variables alpha then beta.
 */
int orc_vforce2(const orc_mesh *m, const int *lm, const int *maskg, const int *mconn, int ncon,
                const int *jcsc, const int *icsc, long long nz, int lisp, int liss, double freq,
                double py, const float *wave, float *fmat)
{
    const double TWOPI = 6.2831853071795862;
    double omega = TWOPI * freq;
    orc_ws w;
    ws_init(&w, m->nord);
    int nen = w.nen, nee = w.nee, nq = w.nq, nint = w.nint;
    const double *wts = w.xigll + nint;
    double *dab1 = (double *)malloc(sizeof(double) * nq), *dab2 = (double *)malloc(sizeof(double) * nq);
    double *dmdb = (double *)malloc(sizeof(double) * nee * nee);
    zc *dkdb = (zc *)malloc(sizeof(zc) * nee * nee);
    int ierr = 0, inpgl = 0;
    for (int p = 0; p < m->nnpg && !ierr; p++) {
        if (maskg[p] <= 0) continue;
        inpgl++;
        int i1 = jcsc[inpgl - 1], i2 = jcsc[inpgl] - 1, nnzrow = i2 - i1 + 1;
        for (int v = 0; v < lisp + liss; v++)
            for (int k = 0; k < 2 * nnzrow; k++) fmat[2 * (size_t)(v * nz + i1 - 1) + k] = 0.0f;
        for (int ic = 0; ic < ncon; ic++) {
            int e = mconn[p + (size_t)m->nnpg * ic];
            if (e <= 0) break;
            ierr = djacab(m, e - 1, p + 1, nen, nint, w.xigll, w.shl, w.det, dab1, dab2, w.shg);
            if (ierr) break;
            dabmkisob25(nen, nint, lisp, liss, omega, py, wts, w.det, dab1, dab2, w.shg, w.me, dmdb,
                        w.ke, dkdb);
            const int *lme = lm + (size_t)3 * nen * (e - 1);
            for (int ipe = 0; ipe < nee; ipe++) {
                int idof = lme[ipe];
                if (idof <= 0) continue;
                int inz = ibsect(nnzrow, idof, icsc + (i1 - 1));
                if (inz <= 0 || inz > nnzrow) { ierr = 3; break; }
                for (int iqe = 0; iqe < nee; iqe++) {
                    int jdof = lme[iqe];
                    if (jdof <= 0) continue;
                    cc wv = cmk(wave[2 * (jdof - 1)], wave[2 * (jdof - 1) + 1]);
                    int v = 0;
                    for (int var = 0; var < 2; var++) {
                        if ((var == 0 && !lisp) || (var == 1 && !liss)) continue;
                        const double *dm = var == 0 ? w.me : dmdb;
                        const zc *dk = var == 0 ? w.ke : dkdb;
                        double ar = dm[ipe + nee * iqe] + dk[ipe + nee * iqe].re;
                        double ai = 0.0 + dk[ipe + nee * iqe].im;
                        cc t = cmulf(cmk((float)ar, (float)ai), wv);
                        float *f = fmat + 2 * ((size_t)v * nz + i1 - 1 + inz - 1);
                        f[0] = f[0] + t.re;
                        f[1] = f[1] + t.im;
                        v++;
                    }
                }
            }
            if (ierr) break;
        }
    }
    free(dab1); free(dab2); free(dmdb); free(dkdb);
    ws_free(&w);
    return ierr;
}

/*
 * MET225_MOD (qpmfree.f90:1000-1250), one process: the Hessian-vector terms
 * of the Gauss-Newton / second-order adjoint inner loop.  For every
 * inversion anchor (MASKG order) and its connected elements (MCONN order),
 * with the DJACAB + DABMKISOB25 matrices C_v = CMPLX(DCMPLX(DMD_v,0) + DKD_v)
 * and CWGHT = CMPLX(SNGL(ELEM_WTS(e)), 0):
 *     T1_v(row) += (CWGHT * C_v(row, col)) * WAVE(col)
 *     T2_v(row) += (CWGHT * C_v(row, col)) * ALPHA(col)
 * in COMPLEX*8.  T1, T2 are nulled inside the element loop
 * (qpmfree.f90:1149-1156), so only the last connected element survives;
 * accumulate = 1 keeps every element.  Then, over the anchor's CSC rows in
 * order, PBUF1(ia35) -= REAL(CONJG(T1_v) * NU), PBUF2(ia35) -=
 * REAL(CONJG(T2_v) * ADJLAM) (qpmfree.f90:1223-1226), ia35 =
 * (inpinv - 1) * nvinv + ivinv, alpha before beta.  The MPI_REDUCE of the
 * buffers is a copy here.  p1buf, p2buf: REAL*4 [nnpinv * nvinv],
 * overwritten.  Vectors: COMPLEX*8 [ndof].
 */
int orc_met225(const orc_mesh *m, const int *lm, const int *maskg, const int *mconn, int ncon,
               const double *elem_wts, const int *jcsc, const int *icsc, int lisp, int liss,
               double freq, double py, const float *adjlam, const float *nu, const float *alpha,
               const float *wave, int accumulate, float *p1buf, float *p2buf)
{
    const double TWOPI = 6.2831853071795862;
    double omega = TWOPI * freq;
    orc_ws w;
    ws_init(&w, m->nord);
    int nen = w.nen, nee = w.nee, nq = w.nq, nint = w.nint, nvinv = lisp + liss;
    const double *wts = w.xigll + nint;
    double *dab1 = (double *)malloc(sizeof(double) * nq), *dab2 = (double *)malloc(sizeof(double) * nq);
    double *dmdb = (double *)malloc(sizeof(double) * nee * nee);
    zc *dkdb = (zc *)malloc(sizeof(zc) * nee * nee);
    int maxrow = 0, nnpinv = 0;
    for (int p = 0; p < m->nnpg; p++)
        if (maskg[p] > 0) nnpinv++;
    for (int k = 0; k < nnpinv; k++)
        if (jcsc[k + 1] - jcsc[k] > maxrow) maxrow = jcsc[k + 1] - jcsc[k];
    cc *t1 = (cc *)malloc(sizeof(cc) * 2 * (maxrow + 1)), *t2 = (cc *)malloc(sizeof(cc) * 2 * (maxrow + 1));
    for (int k = 0; k < nnpinv * nvinv; k++) p1buf[k] = p2buf[k] = 0.0f;
    int ierr = 0, inpgl = 0;
    for (int p = 0; p < m->nnpg && !ierr; p++) {
        if (maskg[p] <= 0) continue;
        inpgl++;
        const int inpinv = maskg[p];
        int i1 = jcsc[inpgl - 1], i2 = jcsc[inpgl] - 1, nnzrow = i2 - i1 + 1;
        for (int k = 0; k < 2 * maxrow; k++) t1[k] = t2[k] = cmk(0.0f, 0.0f);
        for (int ic = 0; ic < ncon; ic++) {
            int e = mconn[p + (size_t)m->nnpg * ic];
            if (e <= 0) break;
            ierr = djacab(m, e - 1, p + 1, nen, nint, w.xigll, w.shl, w.det, dab1, dab2, w.shg);
            if (ierr) break;
            dabmkisob25(nen, nint, lisp, liss, omega, py, wts, w.det, dab1, dab2, w.shg, w.me, dmdb,
                        w.ke, dkdb);
            if (!accumulate)
                for (int k = 0; k < 2 * maxrow; k++) t1[k] = t2[k] = cmk(0.0f, 0.0f);
            cc cwght = cmk((float)elem_wts[e - 1], 0.0f);
            const int *lme = lm + (size_t)3 * nen * (e - 1);
            for (int ipe = 0; ipe < nee; ipe++) {
                int idof = lme[ipe];
                if (idof <= 0) continue;
                int inz = ibsect(nnzrow, idof, icsc + (i1 - 1));
                if (inz <= 0 || inz > nnzrow) { ierr = 3; break; }
                for (int iqe = 0; iqe < nee; iqe++) {
                    int jdof = lme[iqe];
                    if (jdof <= 0) continue;
                    cc wv = cmk(wave[2 * (jdof - 1)], wave[2 * (jdof - 1) + 1]);
                    cc av = cmk(alpha[2 * (jdof - 1)], alpha[2 * (jdof - 1) + 1]);
                    int v = 0;
                    for (int var = 0; var < 2; var++) {
                        if ((var == 0 && !lisp) || (var == 1 && !liss)) continue;
                        const double *dm = var == 0 ? w.me : dmdb;
                        const zc *dk = var == 0 ? w.ke : dkdb;
                        double ar = dm[ipe + nee * iqe] + dk[ipe + nee * iqe].re;
                        double ai = 0.0 + dk[ipe + nee * iqe].im;
                        cc cw = cmulf(cwght, cmk((float)ar, (float)ai));
                        cc a1 = cmulf(cw, wv), a2 = cmulf(cw, av);
                        cc *r1 = &t1[v * maxrow + inz - 1], *r2 = &t2[v * maxrow + inz - 1];
                        r1->re = r1->re + a1.re;
                        r1->im = r1->im + a1.im;
                        r2->re = r2->re + a2.re;
                        r2->im = r2->im + a2.im;
                        v++;
                    }
                }
            }
            if (ierr) break;
        }
        if (ierr) break;
        for (int v = 0; v < nvinv; v++) {
            const int ia35 = (inpinv - 1) * nvinv + v;
            for (int k = 0; k < nnzrow; k++) {
                const int idof = icsc[i1 - 1 + k];
                const cc a = t1[v * maxrow + k], b = t2[v * maxrow + k];
                const float nr = nu[2 * (idof - 1)], ni = nu[2 * (idof - 1) + 1];
                const float lr = adjlam[2 * (idof - 1)], li = adjlam[2 * (idof - 1) + 1];
                const float ar = a.re, ai = -a.im, br = b.re, bi = -b.im; /* CONJG */
                p1buf[ia35] = p1buf[ia35] - (ar * nr - ai * ni);
                p2buf[ia35] = p2buf[ia35] - (br * lr - bi * li);
            }
        }
    }
    free(dab1); free(dab2); free(dmdb); free(dkdb); free(t1); free(t2);
    ws_free(&w);
    return ierr;
}

/*
 * CADJ_NU_ALPHA (qpmfree.f90:622-996), one process, without its two MUMPS
 * solves: the right-hand sides of the second-order adjoint (nu) and of the
 * model-perturbation field (alpha), and the P3 term, for a model
 * perturbation V(NA35).  Per inversion anchor (MASKG order), connected
 * element (MCONN order), row IPE (IDOF > 0), column IQE (JDOF > 0) and
 * variable (alpha before beta), with C_v the DJACAB2 + DABM2KISOB25
 * first-derivative blocks (the same arithmetic as DABMKISOB25; the
 * second-derivative blocks it also forms, CARG2, enter none of the sums) and
 * CWGHT = CMPLX(SNGL(ELEM_WTS(e)) * V(ia35), 0):
 *     RHSBNU(JDOF) += ADJLAM(IDOF) * CONJG(CWGHT * C_v(IPE, IQE))
 *     RHSALP(IDOF) += CWGHT * C_v(IPE, IQE) * WAVE(JDOF)
 *     TEMP_v(row)  += CWGHT * C_v(IPE, IQE) * WAVE(JDOF)
 * TEMP is nulled inside the element loop (qpmfree.f90:823-829: only the last
 * connected element survives; accumulate = 1 keeps every element), then
 * P3(ia35) -= REAL(CONJG(TEMP_v) * ADJLAM) over the anchor's CSC rows.  The
 * solves that follow are the caller's: NU = CONJG(S^-T CONJG(RHSBNU)),
 * ALPHA = S^-1 RHSALP.  Vectors COMPLEX*8 [ndof], v and p3 REAL*4
 * [nnpinv * nvinv]; outputs overwritten.
 */
int orc_cadj_nu_alpha(const orc_mesh *m, const int *lm, int ndof, const int *maskg,
                      const int *mconn, int ncon, const double *elem_wts, const int *jcsc,
                      const int *icsc, int lisp, int liss, double freq, double py,
                      const float *v, const float *adjlam, const float *wave, int accumulate,
                      float *rhsbnu, float *rhsalp, float *p3)
{
    const double TWOPI = 6.2831853071795862;
    double omega = TWOPI * freq;
    orc_ws w;
    ws_init(&w, m->nord);
    int nen = w.nen, nee = w.nee, nq = w.nq, nint = w.nint, nvinv = lisp + liss;
    const double *wts = w.xigll + nint;
    double *dab1 = (double *)malloc(sizeof(double) * nq), *dab2 = (double *)malloc(sizeof(double) * nq);
    double *dmdb = (double *)malloc(sizeof(double) * nee * nee);
    zc *dkdb = (zc *)malloc(sizeof(zc) * nee * nee);
    int maxrow = 0, nnpinv = 0;
    for (int p = 0; p < m->nnpg; p++)
        if (maskg[p] > 0) nnpinv++;
    for (int k = 0; k < nnpinv; k++)
        if (jcsc[k + 1] - jcsc[k] > maxrow) maxrow = jcsc[k + 1] - jcsc[k];
    cc *temp = (cc *)malloc(sizeof(cc) * 2 * (maxrow + 1));
    for (int k = 0; k < 2 * ndof; k++) rhsbnu[k] = rhsalp[k] = 0.0f;
    for (int k = 0; k < nnpinv * nvinv; k++) p3[k] = 0.0f;
    int ierr = 0, inpgl = 0;
    for (int p = 0; p < m->nnpg && !ierr; p++) {
        if (maskg[p] <= 0) continue;
        inpgl++;
        const int inpinv = maskg[p];
        int i1 = jcsc[inpgl - 1], i2 = jcsc[inpgl] - 1, nnzrow = i2 - i1 + 1;
        for (int k = 0; k < 2 * maxrow; k++) temp[k] = cmk(0.0f, 0.0f);
        for (int ic = 0; ic < ncon; ic++) {
            int e = mconn[p + (size_t)m->nnpg * ic];
            if (e <= 0) break;
            ierr = djacab(m, e - 1, p + 1, nen, nint, w.xigll, w.shl, w.det, dab1, dab2, w.shg);
            if (ierr) break;
            dabmkisob25(nen, nint, lisp, liss, omega, py, wts, w.det, dab1, dab2, w.shg, w.me, dmdb,
                        w.ke, dkdb);
            if (!accumulate)
                for (int k = 0; k < 2 * maxrow; k++) temp[k] = cmk(0.0f, 0.0f);
            const float swt = (float)elem_wts[e - 1];
            const int *lme = lm + (size_t)3 * nen * (e - 1);
            for (int ipe = 0; ipe < nee; ipe++) {
                int idof = lme[ipe];
                if (idof <= 0) continue;
                int inz = ibsect(nnzrow, idof, icsc + (i1 - 1));
                if (inz <= 0 || inz > nnzrow) { ierr = 3; break; }
                cc lam = cmk(adjlam[2 * (idof - 1)], adjlam[2 * (idof - 1) + 1]);
                for (int iqe = 0; iqe < nee; iqe++) {
                    int jdof = lme[iqe];
                    if (jdof <= 0) continue;
                    cc wv = cmk(wave[2 * (jdof - 1)], wave[2 * (jdof - 1) + 1]);
                    int vv = 0;
                    for (int var = 0; var < 2; var++) {
                        if ((var == 0 && !lisp) || (var == 1 && !liss)) continue;
                        const double *dm = var == 0 ? w.me : dmdb;
                        const zc *dk = var == 0 ? w.ke : dkdb;
                        double ar = dm[ipe + nee * iqe] + dk[ipe + nee * iqe].re;
                        double ai = 0.0 + dk[ipe + nee * iqe].im;
                        const int ia35 = (inpinv - 1) * nvinv + vv;
                        cc cwght = cmk(swt * v[ia35], 0.0f);
                        cc cw = cmulf(cwght, cmk((float)ar, (float)ai));
                        cc nb = cmulf(lam, cmk(cw.re, -cw.im));
                        rhsbnu[2 * (jdof - 1)] = rhsbnu[2 * (jdof - 1)] + nb.re;
                        rhsbnu[2 * (jdof - 1) + 1] = rhsbnu[2 * (jdof - 1) + 1] + nb.im;
                        cc al = cmulf(cw, wv);
                        rhsalp[2 * (idof - 1)] = rhsalp[2 * (idof - 1)] + al.re;
                        rhsalp[2 * (idof - 1) + 1] = rhsalp[2 * (idof - 1) + 1] + al.im;
                        cc *t = &temp[vv * maxrow + inz - 1];
                        t->re = t->re + al.re;
                        t->im = t->im + al.im;
                        vv++;
                    }
                }
            }
            if (ierr) break;
        }
        if (ierr) break;
        for (int vv = 0; vv < nvinv; vv++) {
            const int ia35 = (inpinv - 1) * nvinv + vv;
            for (int k = 0; k < nnzrow; k++) {
                const int idof = icsc[i1 - 1 + k];
                const cc a = temp[vv * maxrow + k];
                const float lr = adjlam[2 * (idof - 1)], li = adjlam[2 * (idof - 1) + 1];
                const float ar = a.re, ai = -a.im; /* CONJG */
                p3[ia35] = p3[ia35] - (ar * lr - ai * li);
            }
        }
    }
    free(dab1); free(dab2); free(dmdb); free(dkdb); free(temp);
    ws_free(&w);
    return ierr;
}

/*
 * PCHADJ (pchadj.f90:1-330), one process, after its Green's-function solve:
 * for every inversion anchor column and every receiver right-hand side,
 *     JACL(irhs, v) = sum_rows GRNSFNS((irhs-1)*NDOF + JDOF) * FMAT(row, v)
 * in COMPLEX*8 (pchadj.f90:241-246), then the block-diagonal preconditioner
 * update HESSB += REAL(JACL^H JACL) (CGEMM 'C','N' with ALPHA = 1, BETA = 0,
 * summed over irhs in order as the reference BLAS does, then SAXPY,
 * pchadj.f90:274-300, 312-323).  grns: COMPLEX*8 [nrhs][ndof]; fmat:
 * COMPLEX*8 [nvinv][nz]; hessb: REAL*4 [nnpinv * nvinv^2] updated in place,
 * block (col, iv, jv) at (col * nvinv + iv) * nvinv + jv; jacl (nullable):
 * COMPLEX*8 [nnpinv * nvinv][nrhs].
 */
void orc_pchadj(int nnpinv, int nvinv, long long nz, int ndof, int nrhs, const int *jcsc,
                const int *icsc, const float *grns, const float *fmat, float *hessb, float *jacl)
{
    cc *jl = (cc *)malloc(sizeof(cc) * (size_t)nrhs * nvinv);
    for (int col = 0; col < nnpinv; col++) {
        for (int irhs = 0; irhs < nrhs; irhs++)
            for (int v = 0; v < nvinv; v++) {
                cc acc = cmk(0.0f, 0.0f);
                for (int i = jcsc[col]; i <= jcsc[col + 1] - 1; i++) {
                    const int jdof = icsc[i - 1];
                    if (jdof == 0) continue;
                    const size_t jl0 = (size_t)irhs * ndof + jdof - 1;
                    cc g = cmk(grns[2 * jl0], grns[2 * jl0 + 1]);
                    const size_t f0 = (size_t)v * nz + i - 1;
                    cc f = cmk(fmat[2 * f0], fmat[2 * f0 + 1]);
                    cc t = cmulf(g, f);
                    acc.re = acc.re + t.re;
                    acc.im = acc.im + t.im;
                }
                jl[(size_t)irhs * nvinv + v] = acc;
                if (jacl) {
                    jacl[2 * (((size_t)col * nvinv + v) * nrhs + irhs)] = acc.re;
                    jacl[2 * (((size_t)col * nvinv + v) * nrhs + irhs) + 1] = acc.im;
                }
            }
        for (int iv = 0; iv < nvinv; iv++)
            for (int jv = 0; jv < nvinv; jv++) {
                cc temp = cmk(0.0f, 0.0f);
                for (int l = 0; l < nrhs; l++) {
                    cc a = jl[(size_t)l * nvinv + iv], b = jl[(size_t)l * nvinv + jv];
                    cc t = cmulf(cmk(a.re, -a.im), b);
                    temp.re = temp.re + t.re;
                    temp.im = temp.im + t.im;
                }
                cc h = cmulf(cmk(1.0f, 0.0f), temp);
                float hb = 0.0f + h.re;
                float *y = &hessb[((size_t)col * nvinv + iv) * nvinv + jv];
                *y = *y + 1.0f * hb;
            }
    }
    free(jl);
}

/* ADJFLAM_DIST (adjgrad.f90:88-145) followed by GRADL = GRADL - GPROD
 * (adjgrad.f90:76); REAL*4 arithmetic. gradl: [nnpinv], adjlam: COMPLEX*8 */
void orc_adjflam(int nnpinv, const int *jcsc, const int *icsc, const float *fmat,
                 const float *adjlam, float *gradl)
{
    float *vwork = (float *)calloc(nnpinv, sizeof(float));
    for (int k = 0; k < nnpinv; k++) {
        for (int i = jcsc[k]; i <= jcsc[k + 1] - 1; i++) {
            int jdof = icsc[i - 1];
            float fr = fmat[2 * (i - 1)], fi = -fmat[2 * (i - 1) + 1]; /* conj(F) */
            float lr = adjlam[2 * (jdof - 1)], li = adjlam[2 * (jdof - 1) + 1];
            vwork[k] = vwork[k] - (fr * lr - fi * li);
        }
    }
    for (int k = 0; k < nnpinv; k++) gradl[k] = gradl[k] + (-1.0f) * vwork[k];
    free(vwork);
}

/* WTGRAD (gengmask.f90:384-416) */
void orc_wtgrad(int na35, const float *wgrad, float *grad)
{
    for (int i = 0; i < na35; i++) grad[i] = grad[i] * wgrad[i];
}

/* AVGRAD (gengmask.f90:1202-1266), REAL*4; mconn MCONN(NNPG,NCON) and ieng
 * IENG(4,NELEM) column-major, 1-based */
void orc_avgrad(int nnpg, int ncon, int nvinv, int ncasc, const int *maskg, const int *mconn,
                const int *ieng, int na35, float *grad)
{
    if (ncasc <= 0) return;
    float *work = (float *)malloc(sizeof(float) * (size_t)na35);
    for (int icasc = 0; icasc < ncasc; icasc++) {
        memcpy(work, grad, sizeof(float) * (size_t)na35);
        for (int inpg = 1; inpg <= nnpg; inpg++) {
            int inpinv = maskg[inpg - 1];
            if (inpinv <= 0) continue;
            float xavg[2] = {0.0f, 0.0f};
            int navg[2] = {0, 0};
            for (int icon = 1; icon <= ncon; icon++) {
                int ielem = mconn[(inpg - 1) + (size_t)nnpg * (icon - 1)];
                if (ielem == 0) break;
                for (int ia = 1; ia <= 4; ia++) {
                    int jnpg = ieng[4 * (ielem - 1) + ia - 1];
                    if (jnpg == 0) break;
                    int jnpinv = maskg[jnpg - 1];
                    if (jnpinv > 0)
                        for (int iv = 1; iv <= nvinv; iv++) {
                            xavg[iv - 1] = xavg[iv - 1] + grad[(jnpinv - 1) * nvinv + iv - 1];
                            navg[iv - 1] = navg[iv - 1] + 1;
                        }
                }
            }
            for (int iv = 1; iv <= nvinv; iv++)
                if (navg[iv - 1] > 0)
                    work[(inpinv - 1) * nvinv + iv - 1] = xavg[iv - 1] / (float)navg[iv - 1];
        }
        memcpy(grad, work, sizeof(float) * (size_t)na35);
    }
    free(work);
}

/* AVGRAD8 (gengmask.f90:1270-1332), REAL*8 */
void orc_avgrad8(int nnpg, int ncon, int nvinv, int ncasc, const int *maskg, const int *mconn,
                 const int *ieng, int na35, double *grad)
{
    if (ncasc <= 0) return;
    double *work = (double *)malloc(sizeof(double) * (size_t)na35);
    for (int icasc = 0; icasc < ncasc; icasc++) {
        memcpy(work, grad, sizeof(double) * (size_t)na35);
        for (int inpg = 1; inpg <= nnpg; inpg++) {
            int inpinv = maskg[inpg - 1];
            if (inpinv <= 0) continue;
            double xavg[2] = {0.0, 0.0};
            int navg[2] = {0, 0};
            for (int icon = 1; icon <= ncon; icon++) {
                int ielem = mconn[(inpg - 1) + (size_t)nnpg * (icon - 1)];
                if (ielem == 0) break;
                for (int ia = 1; ia <= 4; ia++) {
                    int jnpg = ieng[4 * (ielem - 1) + ia - 1];
                    if (jnpg == 0) break;
                    int jnpinv = maskg[jnpg - 1];
                    if (jnpinv > 0)
                        for (int iv = 1; iv <= nvinv; iv++) {
                            xavg[iv - 1] = xavg[iv - 1] + grad[(jnpinv - 1) * nvinv + iv - 1];
                            navg[iv - 1] = navg[iv - 1] + 1;
                        }
                }
            }
            for (int iv = 1; iv <= nvinv; iv++)
                if (navg[iv - 1] > 0)
                    work[(inpinv - 1) * nvinv + iv - 1] = xavg[iv - 1] / (double)navg[iv - 1];
        }
        memcpy(grad, work, sizeof(double) * (size_t)na35);
    }
    free(work);
}

/* ------------------------------------------------------------------------ */
/* forward misfit and adjoint source                                          */
/* EXRESP25D (locrec2d.f:867-925) -> CROTATE (wrapph.f:178) -> CRESID         */
/* (objfn.f:953-1010) -> COBJ4 (objfn.f:5-172) and BPRESID4 (objfn.f:757-845) */
/* -> RESID_DRHS (adjgrad.f90:448-523) with HDIFFER (adjgrad.f90:528-566).    */
/* Single precision as in the reference.                                      */
/*   sol: COMPLEX*8 [ndof]; mrdof: MRDOF(3,NREC); obs, wghts: (3,NREC)        */
/*   rhs: COMPLEX*8 [ndof] adjoint RHS (conjugated, as handed to the solver)  */
/* returns the source's sum of COBJ4's terms C (not halved)                   */
/* Options (the INV_INFO fields of the reference's .spec file):               */
/*   norm   NORM: 1 L1, 3 Huber, 4 L1/L2 combination, else L2                  */
/*   irestp IRESTP: 1 phase only, 2 amplitude only, else both                 */
/*   ibphase IBPHASE of HDIFFER (0-6)                                         */
/*   eps, thresh  COBJ4's EPS = EPSS*CRESMN and THRESH = THRESHS*CRESMN       */
/*   dtmax  BPRESID4's DTMAX, dtmax_obj COBJ4's DTMAX (L2 only, 0 = off)      */
/* |z| is restated as sqrt(re^2 + im^2) and complex products in the order     */
/* (ac - bd, ad + bc); BPRESID4's EPS is 0 for every norm (objfn.f:795-797),  */
/* as in the reference.                                                       */
/* ------------------------------------------------------------------------ */
static float cabsf_(cc z) { return sqrtf(z.re * z.re + z.im * z.im); }

/* CRESID (objfn.f:953-1010) */
static cc cresid(int irestp, cc obs, cc est)
{
    if (obs.re == 0.0f && obs.im == 0.0f) return cmk(0.0f, 0.0f);
    if (irestp == 1 || irestp == 2) {
        float adata, pdata, aest, pest;
        if (irestp == 2) {
            adata = sqrtf(obs.re * obs.re + obs.im * obs.im);
            pdata = 0.0f;
            aest = sqrtf(est.re * est.re + est.im * est.im);
            pest = 0.0f;
        } else {
            adata = 1.0f;
            pdata = atan2f(obs.im, obs.re);
            aest = 1.0f;
            pest = atan2f(est.im, est.re);
        }
        cc a = cmulf(cmk(adata, 0.0f), cmk(cosf(pdata), sinf(pdata)));
        cc b = cmulf(cmk(aest, 0.0f), cmk(cosf(pest), sinf(pest)));
        return cmk(a.re - b.re, a.im - b.im);
    }
    return cmk(obs.re - est.re, obs.im - est.im);
}

/* wrapped phase difference SPHASE(obs) - SPHASE(est) exceeds dtmax in time */
static int phase_jump(cc obs, cc est, double freq, float dtmax)
{
    const float TWOPI_F = (float)6.283185307179586, PI_F = (float)3.1415926535897931;
    float dphi = atan2f(obs.im, obs.re) - atan2f(est.im, est.re);
    if (dphi < -PI_F) dphi = dphi + TWOPI_F;
    if (dphi > +PI_F) dphi = dphi - TWOPI_F;
    return fabs((double)dphi / ((double)TWOPI_F * freq)) > (double)dtmax;
}

/* HDIFFER (adjgrad.f90:528-566) */
void orc_hdiffer(int ibphase, double freq, float *h)
{
    float omega = (float)(2.0 * 3.1415926535897932384626434 * freq);
    float complex z = 1.0f;
    if (ibphase == 1 || ibphase == 2) {
        z = csqrtf(CMPLXF(0.0f, -omega));
        if (ibphase == 2) z = -z;
    } else if (ibphase == 3 || ibphase == 4) {
        z = csqrtf(CMPLXF(0.0f, omega));
        if (ibphase == 4) z = -z;
    } else if (ibphase == 5) {
        z = CMPLXF(0.0f, omega);
    } else if (ibphase == 6) {
        z = CMPLXF(0.0f, 1.0f);
    }
    h[0] = crealf(z);
    h[1] = cimagf(z);
}

float orc_misfit_opt(int ndof, int nrec, const int *mrdof, const double *yrec, double freq,
                     double py, double azmod, const float *recv, const float *sol,
                     const float *obs, const float *wghts, int norm, int irestp, int ibphase,
                     float eps, float thresh, float dtmax, float dtmax_obj, float *est, float *rhs)
{
    const double TWOPI = 6.2831853071795862;
    double omega = TWOPI * freq;
    float cobj = 0.0f;
    float hf[2];
    orc_hdiffer(ibphase, freq, hf);
    const cc hfact = cmk(hf[0], hf[1]);
    if (rhs) for (int i = 0; i < 2 * ndof; i++) rhs[i] = 0.0f;
    for (int ir = 0; ir < nrec; ir++) {
        float ph = (float)(omega * py * yrec[ir]);
        cc cf = cmk(cosf(ph), sinf(ph));
        cc e3[3], o3[3], er[3];
        for (int i = 0; i < 3; i++) {
            int d = mrdof[3 * ir + i];
            if (d != 0) {
                cc rv = cmk(recv[2 * (3 * ir + i)], recv[2 * (3 * ir + i) + 1]);
                cc sv = cmk(sol[2 * (d - 1)], sol[2 * (d - 1) + 1]);
                e3[i] = cmulf(cmulf(rv, sv), cf);
            } else e3[i] = cmk(0.0f, 0.0f);
            if (est) { est[2 * (3 * ir + i)] = e3[i].re; est[2 * (3 * ir + i) + 1] = e3[i].im; }
            o3[i] = cmk(obs[2 * (3 * ir + i)], obs[2 * (3 * ir + i) + 1]);
        }
        /* rotate estimates into the (N,E,Z) frame */
        float th = (float)azmod * 0.017453292519943295f;
        float ct = cosf(th), st = sinf(th);
        er[0] = cmk(e3[0].re * ct - e3[1].re * st, e3[0].im * ct - e3[1].im * st);
        er[1] = cmk(e3[0].re * st + e3[1].re * ct, e3[0].im * st + e3[1].im * ct);
        er[2] = e3[2];
        /* phase shift back to the (u,v,w) frame (adjgrad.f90:288-292) */
        float ph2 = -(float)(omega * py * yrec[ir]);
        cc cf2 = cmk(cosf(ph2), sinf(ph2));
        cc res[3];
        for (int i = 0; i < 3; i++) {
            res[i] = cmk(0.0f, 0.0f);
            if (o3[i].re == 0.0f && o3[i].im == 0.0f) continue;
            const float w = wghts[3 * ir + i];
            const cc S = cmk(w, 0.0f);
            const float sabs = fabsf(w);
            /* ---- COBJ4 term on the unshifted pair */
            {
                cc dif = cresid(irestp, o3[i], er[i]);
                float c;
                if (norm == 1) {
                    c = cabsf_(cmulf(S, dif));
                } else if (norm == 3) {
                    float arg = cabsf_(cmulf(S, dif));
                    c = arg <= eps ? arg * arg / (2.0f * eps) : arg - eps / 2.0f;
                } else if (norm == 4) {
                    float arg = cabsf_(dif), sd = cabsf_(cmulf(S, dif));
                    c = arg <= thresh ? sd * sd / (2.0f * (eps * eps)) : sd / eps;
                } else {
                    cc cd = cmulf(cmk(dif.re, -dif.im), dif);
                    c = sabs * sabs * cd.re;
                    if (dtmax_obj > 0.0f && phase_jump(o3[i], er[i], freq, dtmax_obj)) {
                        float damp = cabsf_(o3[i]) - cabsf_(er[i]);
                        c = irestp == 1 ? sabs * sabs * 4.0f : sabs * sabs * (damp * damp);
                    }
                }
                cobj = cobj + c;
            }
            /* ---- BPRESID4 residual on the shifted pair (EPS = 0) */
            {
                cc ob = cmulf(o3[i], cf2), es = cmulf(er[i], cf2);
                cc dif = cresid(irestp, ob, es);
                const float e0 = 0.0f;
                if (norm == 1 || (norm == 3 && !(cabsf_(cmulf(S, dif)) <= e0))) {
                    cc num = cmulf(S, dif);  /* CONJG(WEIGHT) = WEIGHT */
                    float den = cabsf_(dif);
                    res[i] = cmk(num.re / den, num.im / den);
                } else if (norm == 3) {
                    res[i] = cmulf(cmk(sabs * sabs / e0, 0.0f), dif);
                } else if (norm == 4) {
                    float eps2 = 0.0f;  /* EPSS * EPS**2 with EPS = 0 */
                    float sd = cabsf_(cmulf(S, dif));
                    float denon = eps2 * sqrtf(1.0f + sd * sd / eps2);
                    res[i] = cmulf(cmk(sabs * sabs / denon, 0.0f), dif);
                } else {
                    res[i] = cmulf(cmk(sabs * sabs, 0.0f), dif);
                    if (dtmax > 0.0f && phase_jump(ob, es, freq, dtmax)) res[i] = cmk(0.0f, 0.0f);
                }
            }
        }
        if (!rhs) continue;
        /* unrotate residual */
        float ct2 = cosf(-th), st2 = sinf(-th);
        cc rr[3];
        rr[0] = cmk(res[0].re * ct2 - res[1].re * st2, res[0].im * ct2 - res[1].im * st2);
        rr[1] = cmk(res[0].re * st2 + res[1].re * ct2, res[0].im * st2 + res[1].im * ct2);
        rr[2] = res[2];
        for (int i = 0; i < 3; i++) {
            int d = mrdof[3 * ir + i];
            if (d <= 0 || d > ndof) continue;
            cc t = cmulf(hfact, rr[i]);
            rhs[2 * (d - 1)] = rhs[2 * (d - 1)] + t.re;
            rhs[2 * (d - 1) + 1] = rhs[2 * (d - 1) + 1] + t.im;
        }
    }
    if (rhs) for (int i = 0; i < ndof; i++) rhs[2 * i + 1] = -rhs[2 * i + 1];
    return cobj;
}

/* the defaults of the reference's .spec file: L2, phase and amplitude, no
 * back-propagation filter, no phase-jump test */
float orc_misfit(int ndof, int nrec, const int *mrdof, const double *yrec, double freq, double py,
                 double azmod, const float *recv, const float *sol, const float *obs,
                 const float *wghts, float *est, float *rhs)
{
    return orc_misfit_opt(ndof, nrec, mrdof, yrec, freq, py, azmod, recv, sol, obs, wghts, 2, 3, 0,
                          0.0f, 0.0f, 0.0f, 0.0f, est, rhs);
}
