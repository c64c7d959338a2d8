/*
 * dnl_oracle.c - CPU restatement of DynELA's explicit hot path (FP64).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the GPU engine.  Nothing in the
 * engine links, loads or calls this file.  Every function cites the reference
 * file:line it restates (paths relative to the DynELA checkout).  The
 * arithmetic follows the reference step by step; the one deliberate
 * difference is the 3x3 symmetric eigen-solver inside the polar
 * decomposition: the reference uses a Cuppen divide-and-conquer routine
 * (Sources/dnlMaths/Eigen3x3.C:454-634) while this file uses cyclic Jacobi
 * rotations (a textbook method, e.g. Golub & Van Loan, Matrix Computations,
 * sec. 8.5).  Both give the same U, ln U and R to rounding.
 */
#include "dnl_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define SQRT23 0.81649658092772603273 /* sqrt(2/3), dnlSqrt23 */
#define SQRT32 1.22474487139158904909 /* sqrt(3/2), dnlSqrt32 */
#define TWO_PI 6.28318530717958647692

static char g_err[256];

static void set_err(const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

const char *orc_last_error(void) { return g_err; }

struct orc_model
{
  int type, npe, dim;
  int axi; /* ElementAxi family (ElQua4NAx); ElQua4N2D is plane strain */
  long nN, nE, nIP;
  double *x, *disp, *mass, *fint;
  double *fu[2], *fv[2], *fa[2]; /* nodal fields; fu[f0] is field0 */
  int f0;
  int8_t *bc;
  double *bcv;
  int32_t *bcf;
  int nfunc;
  int32_t *fnp;
  double **fx, **fy;
  int nmat;
  dnl_material *mat;
  int32_t *emat;
  int32_t *conn;
  double *ip;                                   /* [DNL_IP_NCOMP * nIP] */
  double *detJ, *radius, *dNdx, *rot, *dE;      /* per IP transients */
  double N[8][8], dNdxi[8][8][3], w[8];          /* Gauss tables [ip][node] */
  double t, dt, t_end, up_to;
  long inc;
  int ts_method, ts_freq, stress_method;
  double safety, alphaM, beta, gamma, omegaS;
  int status, bad;
  int polar_route;     /* 0: the reference's C = F^T F route, 1: from H = F - I (orc_set_polar_route) */
  double *pv;          /* power-iteration vector [nN*dim] (Model::_powerIterationEV) */
  double pfmax;        /* Model::_powerIterationFreqMax */
  long piters;         /* total power iterations run */
};

/* ---------------------------------------------------------------- tables */

/* Shape functions and derivatives at the Gauss points, from the closed forms of
 * ElQua4NAx.C:269-297 and ElHex8N3D.C:561-632; the Gauss point g sits at the
 * local coordinates of node g divided by sqrt(3), weight 1
 * (ElQua4NAx.C:64-110, ElHex8N3D.C:94-225). */
static const double NODE_SIGN[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                       {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

static void build_tables(orc_model *m)
{
  const double a = 1.0 / sqrt(3.0);
  for (int g = 0; g < m->npe; g++)
  {
    double xi[3] = {NODE_SIGN[g][0] * a, NODE_SIGN[g][1] * a, NODE_SIGN[g][2] * a};
    m->w[g] = 1.0;
    for (int n = 0; n < m->npe; n++)
    {
      const double *s = NODE_SIGN[n];
      if (m->dim == 2)
      {
        double f0 = 1.0 + s[0] * xi[0], f1 = 1.0 + s[1] * xi[1];
        m->N[g][n] = f0 * f1 / 4.0;
        m->dNdxi[g][n][0] = s[0] * f1 / 4.0;
        m->dNdxi[g][n][1] = s[1] * f0 / 4.0;
        m->dNdxi[g][n][2] = 0.0;
      }
      else
      {
        double f0 = 1.0 + s[0] * xi[0], f1 = 1.0 + s[1] * xi[1], f2 = 1.0 + s[2] * xi[2];
        m->N[g][n] = f0 * f1 * f2 / 8.0;
        m->dNdxi[g][n][0] = s[0] * f1 * f2 / 8.0;
        m->dNdxi[g][n][1] = s[1] * f0 * f2 / 8.0;
        m->dNdxi[g][n][2] = s[2] * f0 * f1 / 8.0;
      }
    }
  }
}

/* ---------------------------------------------------------------- create */

static void *xcalloc(size_t n, size_t sz)
{
  void *p = calloc(n ? n : 1, sz);
  if (!p)
  {
    fprintf(stderr, "oracle: out of memory\n");
    abort();
  }
  return p;
}

orc_model *orc_create(const dnl_model_desc *d)
{
  if (!d || d->n_nodes <= 0 || d->n_elems <= 0 || !d->coords || !d->conn || d->n_materials <= 0 || !d->materials)
  {
    set_err("invalid model description");
    return NULL;
  }
  if (d->elem_type != DNL_ELQUA4NAX && d->elem_type != DNL_ELHEX8N3D && d->elem_type != DNL_ELQUA4N2D)
  {
    set_err("unknown element type %d", d->elem_type);
    return NULL;
  }
  orc_model *m = (orc_model *)xcalloc(1, sizeof(orc_model));
  m->type = d->elem_type;
  m->npe = (m->type == DNL_ELHEX8N3D) ? 8 : 4;
  m->dim = (m->type == DNL_ELHEX8N3D) ? 3 : 2;
  m->axi = (m->type == DNL_ELQUA4NAX);
  m->nN = d->n_nodes;
  m->nE = d->n_elems;
  m->nIP = m->nE * m->npe;
  long n3 = 3 * m->nN;
  m->x = (double *)xcalloc(n3, sizeof(double));
  memcpy(m->x, d->coords, n3 * sizeof(double));
  m->disp = (double *)xcalloc(n3, sizeof(double));
  m->mass = (double *)xcalloc(m->nN, sizeof(double));
  m->fint = (double *)xcalloc(n3, sizeof(double));
  for (int k = 0; k < 2; k++)
  {
    m->fu[k] = (double *)xcalloc(n3, sizeof(double));
    m->fv[k] = (double *)xcalloc(n3, sizeof(double));
    m->fa[k] = (double *)xcalloc(n3, sizeof(double));
  }
  m->conn = (int32_t *)xcalloc(m->nE * m->npe, sizeof(int32_t));
  memcpy(m->conn, d->conn, m->nE * m->npe * sizeof(int32_t));
  for (long k = 0; k < m->nE * m->npe; k++)
    if (m->conn[k] < 0 || m->conn[k] >= m->nN)
    {
      set_err("connectivity entry %ld out of range", k);
      orc_destroy(m);
      return NULL;
    }
  m->nmat = d->n_materials;
  m->mat = (dnl_material *)xcalloc(m->nmat, sizeof(dnl_material));
  memcpy(m->mat, d->materials, m->nmat * sizeof(dnl_material));
  m->emat = (int32_t *)xcalloc(m->nE, sizeof(int32_t));
  if (d->elem_mat)
    memcpy(m->emat, d->elem_mat, m->nE * sizeof(int32_t));
  m->bc = (int8_t *)xcalloc(n3, 1);
  m->bcv = (double *)xcalloc(n3, sizeof(double));
  m->bcf = (int32_t *)xcalloc(n3, sizeof(int32_t));
  for (long k = 0; k < n3; k++)
  {
    m->bc[k] = d->bc_code ? d->bc_code[k] : 0;
    m->bcv[k] = d->bc_value ? d->bc_value[k] : 0.0;
    m->bcf[k] = d->bc_func ? d->bc_func[k] : -1;
    /* an imposed zero speed is a restrain (BoundarySpeed.C:164 skips it, the
       engine and the harness both restrain it) */
    if (m->bc[k] == DNL_BC_SPEED && m->bcv[k] == 0.0)
      m->bc[k] = DNL_BC_RESTRAIN;
  }
  m->nfunc = d->n_functions;
  m->fnp = (int32_t *)xcalloc(m->nfunc, sizeof(int32_t));
  m->fx = (double **)xcalloc(m->nfunc, sizeof(double *));
  m->fy = (double **)xcalloc(m->nfunc, sizeof(double *));
  for (int f = 0; f < m->nfunc; f++)
  {
    int np = d->functions[f].n_points;
    m->fnp[f] = np;
    m->fx[f] = (double *)xcalloc(np, sizeof(double));
    m->fy[f] = (double *)xcalloc(np, sizeof(double));
    memcpy(m->fx[f], d->functions[f].x, np * sizeof(double));
    memcpy(m->fy[f], d->functions[f].y, np * sizeof(double));
  }
  m->ip = (double *)xcalloc((size_t)DNL_IP_NCOMP * m->nIP, sizeof(double));
  m->detJ = (double *)xcalloc(m->nIP, sizeof(double));
  m->radius = (double *)xcalloc(m->nIP, sizeof(double));
  m->dNdx = (double *)xcalloc(m->nIP * m->npe * 3, sizeof(double));
  m->rot = (double *)xcalloc(m->nIP * 9, sizeof(double));
  m->dE = (double *)xcalloc(m->nIP * 6, sizeof(double));
  build_tables(m);

  /* Element::initializeData (Element.C:258-301): T = T0, density = rho0. */
  for (long e = 0; e < m->nE; e++)
  {
    const dnl_material *mt = &m->mat[m->emat[e]];
    for (int g = 0; g < m->npe; g++)
    {
      long q = e * m->npe + g;
      m->ip[DNL_IP_T * m->nIP + q] = mt->T0;
      m->ip[DNL_IP_DENSITY * m->nIP + q] = mt->density;
    }
  }
  /* BoundarySpeed::applyInitial (BoundarySpeed.C:63-73): both fields get the speed. */
  if (d->v_init)
    for (long k = 0; k < n3; k++)
      m->fv[0][k] = m->fv[1][k] = d->v_init[k];
  /* Model::initSolve then applies the constant conditions too (Model.C:429,
     BoundaryCondition.C:131-150, constant after initial): a node under an
     imposed speed takes that condition's whole vector (its imposed components,
     zero elsewhere, before any time function). */
  for (long i = 0; i < m->nN; i++)
  {
    int speed = 0;
    for (int c = 0; c < 3; c++)
      speed |= m->bc[3 * i + c] == DNL_BC_SPEED;
    if (speed)
      for (int c = 0; c < 3; c++)
        m->fv[0][3 * i + c] = m->fv[1][3 * i + c] = m->bc[3 * i + c] == DNL_BC_SPEED ? m->bcv[3 * i + c] : 0.0;
  }
  m->f0 = 0;

  /* Solver settings and Chung-Hulbert parameters (Explicit.C:86-104). */
  double rb = (d->rho_b >= 0.0 && d->rho_b <= 1.0) ? d->rho_b : 0.8182;
  m->alphaM = (2.0 * rb - 1.0) / (1.0 + rb);
  m->beta = (5.0 - 3.0 * rb) / ((1.0 + rb) * (1.0 + rb) * (2.0 - rb));
  m->gamma = 1.5 - m->alphaM;
  m->omegaS = sqrt((12.0 * pow(1.0 + rb, 3) * (2.0 - rb)) / (10.0 + 15.0 * rb - rb * rb + pow(rb, 3) - pow(rb, 4)));
  m->ts_method = d->ts_method;
  m->stress_method = d->stress_method;
  m->ts_freq = d->ts_freq > 0 ? d->ts_freq : 10;
  m->safety = d->ts_safety > 0 ? d->ts_safety : 0.9;
  m->t = d->t_start;
  m->t_end = d->t_end;
  m->up_to = d->t_end;
  return m;
}

void orc_destroy(orc_model *m)
{
  if (!m)
    return;
  free(m->x); free(m->disp); free(m->mass); free(m->fint);
  for (int k = 0; k < 2; k++) { free(m->fu[k]); free(m->fv[k]); free(m->fa[k]); }
  free(m->conn); free(m->mat); free(m->emat); free(m->bc); free(m->bcv); free(m->bcf);
  for (int f = 0; f < m->nfunc; f++) { free(m->fx[f]); free(m->fy[f]); }
  free(m->fnp); free(m->fx); free(m->fy);
  free(m->ip); free(m->detJ); free(m->radius); free(m->dNdx); free(m->rot); free(m->dE);
  free(m->pv);
  free(m);
}

/* ------------------------------------------------------- small tensor maths */

/* symmetric index of (i, j) in the xx, xy, xz, yy, yz, zz storage */
static const int SYM[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};

/* Cyclic Jacobi eigen-decomposition of a symmetric 3x3 matrix a (xx, xy, xz,
 * yy, yz, zz).  Columns of vec are the eigenvectors. */
void orc_sym_eigen3(const double a6[6], double lambda[3], double vec[3][3])
{
  double A[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
    {
      A[i][j] = a6[SYM[i][j]];
      vec[i][j] = (i == j) ? 1.0 : 0.0;
    }
  static const int P[3] = {0, 0, 1}, Q[3] = {1, 2, 2};
  for (int sweep = 0; sweep < 50; sweep++)
  {
    double off = fabs(A[0][1]) + fabs(A[0][2]) + fabs(A[1][2]);
    double diag = fabs(A[0][0]) + fabs(A[1][1]) + fabs(A[2][2]);
    if (off == 0.0 || off <= 1e-18 * diag)
      break;
    for (int k = 0; k < 3; k++)
    {
      int p = P[k], q = Q[k];
      double apq = A[p][q];
      if (apq == 0.0)
        continue;
      double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
      double t;
      if (fabs(theta) > 1e150)
        t = 0.5 / theta;
      else
        t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
      double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
      for (int r = 0; r < 3; r++)
      {
        /* A <- A J (columns p, q) */
        double arp = A[r][p], arq = A[r][q];
        A[r][p] = c * arp - s * arq;
        A[r][q] = s * arp + c * arq;
      }
      for (int r = 0; r < 3; r++)
      {
        /* A <- J^T A (rows p, q) */
        double apr = A[p][r], aqr = A[q][r];
        A[p][r] = c * apr - s * aqr;
        A[q][r] = s * apr + c * aqr;
      }
      A[p][q] = A[q][p] = 0.0;
      for (int r = 0; r < 3; r++)
      {
        double vrp = vec[r][p], vrq = vec[r][q];
        vec[r][p] = c * vrp - s * vrq;
        vec[r][q] = s * vrp + c * vrq;
      }
    }
  }
  for (int i = 0; i < 3; i++)
    lambda[i] = A[i][i];
}

/* Tensor2::polarCuppenLnU (Tensor2.C:1442-1457): C = F^T F (buildFTF,
 * :1315-1328), eigenpairs of C, then polarExtractLnU (:1237-1313):
 * U = sum sqrt(l) n n, U^-1 by cofactors, R = F U^-1, ln U = sum ln(l)/2 n n. */
void orc_polar_lnU(const double F[9], double lnU[6], double R[9])
{
  double C[6];
  C[0] = F[0] * F[0] + F[3] * F[3] + F[6] * F[6];
  C[1] = F[0] * F[1] + F[3] * F[4] + F[6] * F[7];
  C[2] = F[0] * F[2] + F[3] * F[5] + F[6] * F[8];
  C[3] = F[1] * F[1] + F[4] * F[4] + F[7] * F[7];
  C[4] = F[1] * F[2] + F[4] * F[5] + F[7] * F[8];
  C[5] = F[2] * F[2] + F[5] * F[5] + F[8] * F[8];
  double l[3], V[3][3];
  orc_sym_eigen3(C, l, V);
  double P[3][6];
  for (int k = 0; k < 3; k++)
  {
    P[k][0] = V[0][k] * V[0][k];
    P[k][1] = V[0][k] * V[1][k];
    P[k][2] = V[0][k] * V[2][k];
    P[k][3] = V[1][k] * V[1][k];
    P[k][4] = V[1][k] * V[2][k];
    P[k][5] = V[2][k] * V[2][k];
  }
  double sq[3] = {sqrt(l[0]), sqrt(l[1]), sqrt(l[2])};
  double U[6];
  for (int c = 0; c < 6; c++)
    U[c] = sq[0] * P[0][c] + sq[1] * P[1][c] + sq[2] * P[2][c];
  /* inverse of the symmetric U by cofactors */
  double c00 = U[3] * U[5] - U[4] * U[4];
  double c01 = U[2] * U[4] - U[1] * U[5];
  double c02 = U[1] * U[4] - U[2] * U[3];
  double det = U[0] * c00 + U[1] * c01 + U[2] * c02;
  double Ui[6];
  Ui[0] = c00 / det;
  Ui[1] = c01 / det;
  Ui[2] = c02 / det;
  Ui[3] = (U[0] * U[5] - U[2] * U[2]) / det;
  Ui[4] = (U[2] * U[1] - U[0] * U[4]) / det;
  Ui[5] = (U[0] * U[3] - U[1] * U[1]) / det;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      R[3 * i + j] = F[3 * i] * Ui[SYM[0][j]] + F[3 * i + 1] * Ui[SYM[1][j]] + F[3 * i + 2] * Ui[SYM[2][j]];
  double hl[3] = {log(l[0]) / 2, log(l[1]) / 2, log(l[2]) / 2};
  for (int c = 0; c < 6; c++)
    lnU[c] = hl[0] * P[0][c] + hl[1] * P[1][c] + hl[2] * P[2][c];
}

/* The same decomposition from H = F - I without forming C = F^T F: the
 * eigenpairs of A = C - I = H + H^T + H^T H, ln U = sum log1p(mu)/2 n n,
 * U^-1 = I + sum ((1 + mu)^-1/2 - 1) n n, R = F U^-1.  Mathematically the
 * reference's route; numerically the entries of C are 1 + O(strain) and
 * their rounding (about 1e-16 absolute) is a relative error of
 * 1e-16 / strain increment in ln U, which this route does not make (the
 * engine's polar_lnU works on A too).  Test infrastructure: the yardstick of
 * the engine where the strain increments are small (first increments of the
 * quasi-static necking pulls, about 1e-7 per increment). */
void orc_polar_lnU_h(const double H[9], double lnU[6], double R[9])
{
  double A[6];
  A[0] = 2 * H[0] + H[0] * H[0] + H[3] * H[3] + H[6] * H[6];
  A[1] = H[1] + H[3] + H[0] * H[1] + H[3] * H[4] + H[6] * H[7];
  A[2] = H[2] + H[6] + H[0] * H[2] + H[3] * H[5] + H[6] * H[8];
  A[3] = 2 * H[4] + H[1] * H[1] + H[4] * H[4] + H[7] * H[7];
  A[4] = H[5] + H[7] + H[1] * H[2] + H[4] * H[5] + H[7] * H[8];
  A[5] = 2 * H[8] + H[2] * H[2] + H[5] * H[5] + H[8] * H[8];
  double mu[3], V[3][3];
  orc_sym_eigen3(A, mu, V);
  double P[3][6];
  for (int k = 0; k < 3; k++)
  {
    P[k][0] = V[0][k] * V[0][k];
    P[k][1] = V[0][k] * V[1][k];
    P[k][2] = V[0][k] * V[2][k];
    P[k][3] = V[1][k] * V[1][k];
    P[k][4] = V[1][k] * V[2][k];
    P[k][5] = V[2][k] * V[2][k];
  }
  double hl[3], g[3];
  for (int k = 0; k < 3; k++)
  {
    hl[k] = log1p(mu[k]) / 2;
    g[k] = 1.0 / sqrt(1.0 + mu[k]) - 1.0;
  }
  double Wm[6];
  for (int c = 0; c < 6; c++)
  {
    lnU[c] = hl[0] * P[0][c] + hl[1] * P[1][c] + hl[2] * P[2][c];
    Wm[c] = g[0] * P[0][c] + g[1] * P[1][c] + g[2] * P[2][c];
  }
  /* R = (I + H)(I + Wm) = I + H + Wm + H Wm */
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
    {
      double s = H[3 * i + j] + Wm[SYM[i][j]];
      for (int k = 0; k < 3; k++)
        s += H[3 * i + k] * Wm[SYM[k][j]];
      R[3 * i + j] = s + (i == j ? 1.0 : 0.0);
    }
}

void orc_set_polar_route(orc_model *m, int route) { m->polar_route = route; }

/* SymTensor2::dotRxRT (SymTensor2.C:512-523): R S R^T. */
static void rot_sym(const double R[9], double S[6])
{
  double out[6];
  for (int i = 0; i < 3; i++)
    for (int j = i; j < 3; j++)
    {
      double s = 0.0;
      for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++)
          s += R[3 * i + k] * S[SYM[k][l]] * R[3 * j + l];
      out[SYM[i][j]] = s;
    }
  memcpy(S, out, sizeof(out));
}

static double sym_norm(const double s[6]) /* SymTensor2::norm, SymTensor2.h:362-367 */
{
  return sqrt(s[0] * s[0] + s[3] * s[3] + s[5] * s[5] + 2.0 * (s[1] * s[1] + s[2] * s[2] + s[4] * s[4]));
}

static double sym_ddot(const double a[6], const double b[6]) /* SymTensor2::doubleDot, SymTensor2.C:640-649 */
{
  return a[0] * b[0] + a[3] * b[3] + a[5] * b[5] + 2.0 * (a[1] * b[1] + a[2] * b[2] + a[4] * b[4]);
}

/* ----------------------------------------------------------- Johnson-Cook */

/* JohnsonCookLaw::getYieldStress (JohnsonCookLaw.C:146-170). */
double orc_jc_yield(const dnl_material *p, double epsp, double depsp, double T)
{
  double hard = p->A + p->B * pow(epsp, p->n);
  double visc = (depsp > p->depsp0) ? 1.0 + p->C * log(depsp / p->depsp0) : 1.0;
  double temp = 1.0;
  if (T > p->Tref)
    temp = (T < p->Tm) ? 1.0 - pow((T - p->Tref) / (p->Tm - p->Tref), p->m) : 0.0;
  return hard * visc * temp;
}

/* JohnsonCookLaw::getDerivateYieldStress (JohnsonCookLaw.C:298-339). */
double orc_jc_hardening(const dnl_material *p, double epsp, double depsp, double T, double dt)
{
  double temp1 = 0.0;
  double hard0 = p->A + p->B * pow(epsp, p->n);
  double visc0 = (depsp > p->depsp0) ? 1.0 + p->C * log(depsp / p->depsp0) : 1.0;
  double temp0 = 1.0;
  if (T > p->Tref)
  {
    if (T < p->Tm)
    {
      temp1 = pow((T - p->Tref) / (p->Tm - p->Tref), p->m);
      temp0 = 1.0 - temp1;
    }
    else
      temp0 = 0.0;
  }
  double h = p->n * p->B * pow(epsp, p->n - 1.0) * visc0 * temp0;
  if (depsp > p->depsp0)
    h += hard0 * p->C * temp0 / (depsp * dt);
  if (T > p->Tref && T < p->Tm)
    h -= p->m * p->taylor_quinney * hard0 * hard0 * visc0 * visc0 * temp0 * temp1 /
         (p->density * p->heat_capacity * (T - p->Tref));
  return h;
}

/* -------------------------------------------------------- radial return */

int orc_radial_return_method(const dnl_material *mat, const double dE[6], double dt, double *st, int direct);

enum { RS_S = 0, RS_EP = 6, RS_EPSP = 12, RS_DEPSP, RS_GAMMA, RS_GCUM, RS_YIELD, RS_T, RS_P, RS_EINT, RS_EINEL, RS_N };

/* Element::computeStress (Element.C:407-622) for one integration point, or
 * with direct != 0 Element::computeStressDirect (Element.C:625-850): one
 * step gamma = (|s*| - sqrt(2/3) sigma_y) / (2G (1 + h / (3G))) with the
 * slope h at the previous plastic strain and rate and the initial temperature,
 * then the yield stress at the new state. */
int orc_radial_return_method(const dnl_material *mat, const double dE[6], double dt, double *st, int direct)
{
  const double gammaInitial = 1e-8, tolNR = 1e-8;
  const int itMax = 250;
  double TwoG = mat->young / (1.0 + mat->poisson); /* Material.h:110-114 */
  double TwoG32 = SQRT32 * TwoG;
  double heatFrac = mat->taylor_quinney / (mat->density * mat->heat_capacity);
  double sOld[6], dev[6];
  memcpy(sOld, st + RS_S, sizeof(sOld));
  double p0 = (sOld[0] + sOld[3] + sOld[5]) / 3.0;
  memcpy(dev, sOld, sizeof(dev));
  dev[0] -= p0;
  dev[3] -= p0;
  dev[5] -= p0;
  double Snorm0 = sym_norm(dev);
  double pe = (dE[0] + dE[3] + dE[5]) / 3.0;
  double dEd[6] = {dE[0] - pe, dE[1], dE[2], dE[3] - pe, dE[4], dE[5] - pe};
  for (int c = 0; c < 6; c++)
    dev[c] += TwoG * dEd[c];
  double Snorm = sym_norm(dev);
  double Strial = SQRT32 * Snorm;
  double T0 = st[RS_T], T = T0;
  double plasticStrain = st[RS_EPSP];
  double plasticStrainRate = st[RS_DEPSP];
  double gamma = 0.0;
  double yield = st[RS_YIELD];
  int iterate = 0;
  (void)plasticStrainRate;
  if (yield == 0.0)
  {
    yield = orc_jc_yield(mat, gammaInitial, gammaInitial / dt, T);
    st[RS_YIELD] = yield;
  }
  if (Strial > yield && direct)
  {
    double hard = orc_jc_hardening(mat, plasticStrain > 0.0 ? plasticStrain : gammaInitial, plasticStrainRate, T, dt);
    gamma = (Snorm - SQRT23 * yield) / (TwoG * (1.0 + hard / (1.5 * TwoG)));
    plasticStrainRate = SQRT23 * gamma / dt;
    plasticStrain = st[RS_EPSP] + SQRT23 * gamma;
    T = T0 + 0.5 * gamma * heatFrac * (SQRT23 * yield + Snorm0);
    yield = orc_jc_yield(mat, plasticStrain, plasticStrainRate, T);
    for (int c = 0; c < 6; c++)
      st[RS_EP + c] += gamma * dev[c] / Snorm;
    double scale = 1.0 - TwoG * gamma / Snorm;
    for (int c = 0; c < 6; c++)
      dev[c] *= scale;
    st[RS_EPSP] += SQRT23 * gamma;
    st[RS_DEPSP] = SQRT23 * gamma / dt;
    st[RS_GAMMA] = gamma;
    st[RS_GCUM] += gamma;
    st[RS_YIELD] = yield;
  }
  else if (Strial > yield)
  {
    double gammaMin = 0.0;
    double gammaMax = (Strial - yield) / TwoG32;
    gamma = st[RS_GAMMA];
    if (plasticStrain == 0.0)
      gamma = SQRT32 * gammaInitial;
    plasticStrainRate = SQRT23 * gamma / dt;
    plasticStrain = st[RS_EPSP] + SQRT23 * gamma;
    T = T0 + 0.5 * gamma * heatFrac * (SQRT23 * yield + Snorm0);
    for (;;)
    {
      yield = orc_jc_yield(mat, plasticStrain, plasticStrainRate, T);
      double fun = Strial - gamma * TwoG32 - yield;
      if (fun < 0.0)
        gammaMax = gamma;
      else
        gammaMin = gamma;
      double hard = orc_jc_hardening(mat, plasticStrain, plasticStrainRate, T, dt);
      double dfun = TwoG32 + SQRT23 * hard;
      double dgamma = fun / dfun;
      gamma += dgamma;
      if ((gammaMax - gamma) * (gamma - gammaMin) < 0.0)
      {
        dgamma = 0.5 * (gammaMax - gammaMin);
        gamma = gammaMin + dgamma;
      }
      if (fabs(dgamma) < tolNR)
        break;
      plasticStrainRate = SQRT23 * gamma / dt;
      plasticStrain = st[RS_EPSP] + SQRT23 * gamma;
      T = T0 + 0.5 * gamma * heatFrac * (SQRT23 * yield + Snorm0);
      iterate += 1;
      if (iterate > itMax)
        return -1;
    }
    for (int c = 0; c < 6; c++)
      st[RS_EP + c] += gamma * dev[c] / Snorm;
    double scale = 1.0 - TwoG * gamma / Snorm;
    for (int c = 0; c < 6; c++)
      dev[c] *= scale;
    st[RS_EPSP] += SQRT23 * gamma;
    st[RS_DEPSP] = SQRT23 * gamma / dt;
    st[RS_GAMMA] = gamma;
    st[RS_GCUM] += gamma;
    st[RS_YIELD] = yield;
  }
  double p = st[RS_P];
  double sNew[6] = {dev[0] + p, dev[1], dev[2], dev[3] + p, dev[4], dev[5] + p};
  memcpy(st + RS_S, sNew, sizeof(sNew));
  double sum[6];
  for (int c = 0; c < 6; c++)
    sum[c] = sOld[c] + sNew[c];
  st[RS_EINT] += 0.5 * sym_ddot(dE, sum) / mat->density;
  if (gamma != 0.0)
  {
    double plWorkInc = 0.5 * gamma * (sym_norm(dev) + Snorm0);
    st[RS_EINEL] += plWorkInc / mat->density;
    st[RS_T] += heatFrac * plWorkInc;
  }
  return iterate;
}

int orc_radial_return(const dnl_material *mat, const double dE[6], double dt, double *st)
{
  return orc_radial_return_method(mat, dE, dt, st, 0);
}

/* ----------------------------------------------------------- element pass */

#define IPV(m, c, q) (m)->ip[(long)(c) * (m)->nIP + (q)]

/* ElementPlane::computeJacobian (ElementPlane.C:46-102) and
 * Element3D::computeJacobian (Element3D.C:64-115) with the radius of
 * ElementAxi::getRadiusAtIntegrationPoint (ElementAxi.C:46-59). */
static int jacobian(orc_model *m, int reference)
{
  int d = m->dim, npe = m->npe;
  for (long e = 0; e < m->nE; e++)
  {
    const int32_t *cn = m->conn + e * npe;
    for (int g = 0; g < npe; g++)
    {
      long q = e * npe + g;
      double J[3][3] = {{0}};
      for (int n = 0; n < npe; n++)
        for (int i = 0; i < d; i++)
          for (int j = 0; j < d; j++)
            J[i][j] += m->dNdxi[g][n][j] * m->x[3 * cn[n] + i];
      double det, inv[3][3] = {{0}};
      if (d == 2)
      {
        det = J[0][0] * J[1][1] - J[1][0] * J[0][1];
        inv[0][0] = J[1][1] / det;
        inv[0][1] = -J[0][1] / det;
        inv[1][0] = -J[1][0] / det;
        inv[1][1] = J[0][0] / det;
      }
      else
      {
        double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
        double c01 = J[0][2] * J[2][1] - J[0][1] * J[2][2];
        double c02 = J[0][1] * J[1][2] - J[0][2] * J[1][1];
        det = J[0][0] * c00 + J[1][0] * c01 + J[2][0] * c02;
        inv[0][0] = c00 / det;
        inv[0][1] = c01 / det;
        inv[0][2] = c02 / det;
        inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
        inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
        inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
        inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
        inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
        inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
      }
      if (det < 0.0)
      {
        m->status = DNL_ERR_NEG_JACOBIAN;
        m->bad = (int)e;
        return DNL_ERR_NEG_JACOBIAN;
      }
      m->detJ[q] = det;
      double *dn = m->dNdx + q * npe * 3;
      for (int n = 0; n < npe; n++)
        for (int k = 0; k < d; k++)
        {
          double s = 0.0;
          for (int j = 0; j < d; j++)
            s += m->dNdxi[g][n][j] * inv[j][k];
          dn[3 * n + k] = s;
        }
      if (m->axi)
      {
        double r = 0.0;
        for (int n = 0; n < npe; n++)
          r += m->N[g][n] * m->x[3 * cn[n]];
        m->radius[q] = r;
      }
      else
        m->radius[q] = 1.0;
      if (reference)
        IPV(m, DNL_IP_DETJ0, q) = (m->axi) ? det * m->radius[q] : det;
    }
  }
  return DNL_OK;
}

/* Element::computeStrains (Element.C:1103-1122) with the deformation gradient
 * of ElementAxi.C:78-100 / Element3D.C:172-195, built from field0->u. */
static void strains(orc_model *m)
{
  int npe = m->npe;
  const double *u = m->fu[m->f0];
  for (long e = 0; e < m->nE; e++)
  {
    const int32_t *cn = m->conn + e * npe;
    for (int g = 0; g < npe; g++)
    {
      long q = e * npe + g;
      const double *dn = m->dNdx + q * npe * 3;
      /* the reference sums the gradient into F = I; the H route sums it from
         zero (H = F - I without the rounding of the identity's 1) */
      const double one = m->polar_route ? 0.0 : 1.0;
      double H[9] = {one, 0, 0, 0, one, 0, 0, 0, one};
      if (m->dim == 2)
      {
        double Vr = 0.0;
        for (int n = 0; n < npe; n++)
        {
          const double *un = u + 3 * cn[n];
          H[0] += dn[3 * n] * un[0];
          H[1] += dn[3 * n + 1] * un[0];
          H[3] += dn[3 * n] * un[1];
          H[4] += dn[3 * n + 1] * un[1];
          Vr += m->N[g][n] * un[0];
        }
        if (m->axi)
          H[8] += Vr / m->radius[q];
      }
      else
      {
        for (int n = 0; n < npe; n++)
        {
          const double *un = u + 3 * cn[n];
          for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
              H[3 * i + j] += dn[3 * n + j] * un[i];
        }
      }
      double *de = m->dE + q * 6, *R = m->rot + q * 9;
      if (m->polar_route)
        orc_polar_lnU_h(H, de, R);
      else
        orc_polar_lnU(H, de, R); /* H holds F here */
      for (int c = 0; c < 6; c++)
        IPV(m, DNL_IP_STRAIN + c, q) += de[c];
    }
  }
}

/* Element::computePressure (Element.C:1125-1143). */
static void pressure(orc_model *m)
{
  for (long e = 0; e < m->nE; e++)
  {
    const dnl_material *mt = &m->mat[m->emat[e]];
    double K = mt->young / (3.0 * (1.0 - 2.0 * mt->poisson)); /* Material.h:152-156 */
    double inc = 0.0;
    for (int g = 0; g < m->npe; g++)
    {
      const double *de = m->dE + (e * m->npe + g) * 6;
      inc += de[0] + de[3] + de[5];
    }
    inc /= m->npe;
    for (int g = 0; g < m->npe; g++)
    {
      long q = e * m->npe + g;
      double tr = (IPV(m, 0, q) + IPV(m, 3, q) + IPV(m, 5, q)) / 3.0;
      IPV(m, DNL_IP_PRESSURE, q) = tr + K * inc;
    }
  }
}

/* Model::computeStress (Model.C:837-851) -> Element::computeStress. */
static int stress(orc_model *m, double dt)
{
  double st[RS_N];
  for (long e = 0; e < m->nE; e++)
  {
    const dnl_material *mt = &m->mat[m->emat[e]];
    for (int g = 0; g < m->npe; g++)
    {
      long q = e * m->npe + g;
      for (int c = 0; c < 6; c++)
      {
        st[RS_S + c] = IPV(m, DNL_IP_STRESS + c, q);
        st[RS_EP + c] = IPV(m, DNL_IP_PLASTIC_STRAIN + c, q);
      }
      st[RS_EPSP] = IPV(m, DNL_IP_EPSP, q);
      st[RS_DEPSP] = IPV(m, DNL_IP_DEPSP, q);
      st[RS_GAMMA] = IPV(m, DNL_IP_GAMMA, q);
      st[RS_GCUM] = IPV(m, DNL_IP_GAMMA_CUM, q);
      st[RS_YIELD] = IPV(m, DNL_IP_YIELD, q);
      st[RS_T] = IPV(m, DNL_IP_T, q);
      st[RS_P] = IPV(m, DNL_IP_PRESSURE, q);
      st[RS_EINT] = IPV(m, DNL_IP_EINT, q);
      st[RS_EINEL] = IPV(m, DNL_IP_EINEL, q);
      if (orc_radial_return_method(mt, m->dE + q * 6, dt, st, m->stress_method == DNL_STRESS_DIRECT) < 0)
      {
        m->status = DNL_ERR_NEWTON;
        m->bad = (int)q;
        return DNL_ERR_NEWTON;
      }
      for (int c = 0; c < 6; c++)
      {
        IPV(m, DNL_IP_STRESS + c, q) = st[RS_S + c];
        IPV(m, DNL_IP_PLASTIC_STRAIN + c, q) = st[RS_EP + c];
      }
      IPV(m, DNL_IP_EPSP, q) = st[RS_EPSP];
      IPV(m, DNL_IP_DEPSP, q) = st[RS_DEPSP];
      IPV(m, DNL_IP_GAMMA, q) = st[RS_GAMMA];
      IPV(m, DNL_IP_GAMMA_CUM, q) = st[RS_GCUM];
      IPV(m, DNL_IP_YIELD, q) = st[RS_YIELD];
      IPV(m, DNL_IP_T, q) = st[RS_T];
      IPV(m, DNL_IP_EINT, q) = st[RS_EINT];
      IPV(m, DNL_IP_EINEL, q) = st[RS_EINEL];
    }
  }
  return DNL_OK;
}

/* Element::computeFinalRotation (Element.C:1146-1161). */
static void final_rotation(orc_model *m)
{
  double s[6];
  for (long q = 0; q < m->nIP; q++)
  {
    const double *R = m->rot + q * 9;
    for (int base = 0; base < 18; base += 6)
    {
      for (int c = 0; c < 6; c++)
        s[c] = IPV(m, base + c, q);
      rot_sym(R, s);
      for (int c = 0; c < 6; c++)
        IPV(m, base + c, q) = s[c];
    }
  }
}

/* Element::computeInternalForces (Element.C:362-404) and the element-order
 * scatter-add of Model::computeInternalForces (Model.C:864-899). */
static void internal_forces(orc_model *m)
{
  int d = m->dim, npe = m->npe;
  memset(m->fint, 0, 3 * m->nN * sizeof(double));
  double fe[24];
  for (long e = 0; e < m->nE; e++)
  {
    memset(fe, 0, sizeof(fe));
    for (int g = 0; g < npe; g++)
    {
      long q = e * npe + g;
      double WxdJ = m->w[g] * m->detJ[q];
      if (m->axi)
        WxdJ *= TWO_PI * m->radius[q];
      const double *dn = m->dNdx + q * npe * 3;
      for (int n = 0; n < npe; n++)
      {
        for (int i = 0; i < d; i++)
          for (int j = 0; j < d; j++)
            fe[n * d + i] -= dn[3 * n + j] * IPV(m, SYM[j][i], q) * WxdJ;
        if (m->axi)
          fe[n * d] -= m->N[g][n] * IPV(m, 5, q) / m->radius[q] * WxdJ;
      }
    }
    const int32_t *cn = m->conn + e * npe;
    for (int n = 0; n < npe; n++)
      for (int i = 0; i < d; i++)
        m->fint[3 * cn[n] + i] += fe[n * d + i];
  }
}

static int element_pass(orc_model *m, double dt)
{
  strains(m);
  pressure(m);
  int rc = stress(m, dt);
  if (rc)
    return rc;
  final_rotation(m);
  internal_forces(m);
  return DNL_OK;
}

/* Element::computeDensity (Element.C:1243-1256). */
static void density(orc_model *m)
{
  for (long e = 0; e < m->nE; e++)
  {
    const dnl_material *mt = &m->mat[m->emat[e]];
    for (int g = 0; g < m->npe; g++)
    {
      long q = e * m->npe + g;
      double r = mt->density * IPV(m, DNL_IP_DETJ0, q) / m->detJ[q];
      if (m->axi)
        r /= m->radius[q];
      IPV(m, DNL_IP_DENSITY, q) = r;
    }
  }
}

/* Model::computeMassMatrix (Model.C:537-592) with Element::computeMassMatrix
 * (Element.C:304-339): lumped rho0 N w detJ (2 pi r), assembled in element order. */
static void mass_matrix(orc_model *m)
{
  memset(m->mass, 0, m->nN * sizeof(double));
  double me[8];
  for (long e = 0; e < m->nE; e++)
  {
    const dnl_material *mt = &m->mat[m->emat[e]];
    memset(me, 0, sizeof(me));
    for (int g = 0; g < m->npe; g++)
    {
      long q = e * m->npe + g;
      double WxdJ = m->w[g] * m->detJ[q];
      if (m->axi)
        WxdJ *= TWO_PI * m->radius[q];
      for (int n = 0; n < m->npe; n++)
        me[n] += mt->density * m->N[g][n] * WxdJ;
    }
    for (int n = 0; n < m->npe; n++)
      m->mass[m->conn[e * m->npe + n]] += me[n];
  }
}

/* --------------------------------------------------------------- time step */

/* ElQua4NAx::getCharacteristicLength (ElQua4NAx.C:312-321). */
static double charlen_q4(const double *x, const int32_t *cn)
{
  const double *p0 = x + 3 * cn[0], *p1 = x + 3 * cn[1], *p2 = x + 3 * cn[2], *p3 = x + 3 * cn[3];
  double x31 = p2[0] - p0[0], x24 = p1[0] - p3[0], y42 = p3[1] - p1[1], y31 = p2[1] - p0[1];
  return (x31 * y42 + x24 * y31) / sqrt(2.0 * (x24 * x24 + y42 * y42 + x31 * x31 + y31 * y31));
}

static void sub3(const double *a, const double *b, double *o)
{
  o[0] = a[0] - b[0];
  o[1] = a[1] - b[1];
  o[2] = a[2] - b[2];
}
static void cross3(const double *a, const double *b, double *o)
{
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
static double norm3(const double *a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

/* Area of the quadrilateral face p1 p2 p3 p4 as half the cross product of its
 * diagonals (the AERT formula of ElHex8N3D.C:592-614). */
static double quad_area(const double *p1, const double *p2, const double *p3, const double *p4)
{
  double d1[3], d2[3], c[3];
  sub3(p1, p3, d1);
  sub3(p2, p4, d2);
  cross3(d1, d2, c);
  return 0.5 * norm3(c);
}

/* ElHex8N3D::getVolume (ElHex8N3D.C:651-686): three pyramids with apex at
 * node 7 over the faces 0123, 0154 and 1265. */
static double hex_volume(const double *P[8])
{
  static const int base[3][4] = {{0, 1, 2, 3}, {0, 1, 5, 4}, {1, 2, 6, 5}};
  double vol = 0.0;
  for (int k = 0; k < 3; k++)
  {
    const double *a = P[base[k][0]], *b = P[base[k][1]], *c = P[base[k][2]], *dd = P[base[k][3]];
    double ab[3], ac[3], ad[3], c1[3], c2[3], nrm[3], h[3];
    sub3(b, a, ab);
    sub3(c, a, ac);
    sub3(dd, a, ad);
    cross3(ab, ac, c1);
    cross3(ad, ac, c2);
    double area = (norm3(c1) + norm3(c2)) / 2.0;
    cross3(ab, ad, nrm);
    double nn = norm3(nrm);
    nrm[0] /= nn;
    nrm[1] /= nn;
    nrm[2] /= nn;
    sub3(P[7], a, h);
    double height = fabs(nrm[0] * h[0] + nrm[1] * h[1] + nrm[2] * h[2]);
    vol += area * height / 3.0;
  }
  return vol;
}

/* ElHex8N3D::getCharacteristicLength (ElHex8N3D.C:634-649): volume over the
 * largest face area. */
static double charlen_hex(const double *x, const int32_t *cn)
{
  const double *P[8];
  for (int n = 0; n < 8; n++)
    P[n] = x + 3 * cn[n];
  static const int faces[6][4] = {{0, 1, 2, 3}, {0, 1, 5, 4}, {1, 2, 6, 5}, {3, 2, 6, 7}, {0, 3, 7, 4}, {4, 5, 6, 7}};
  double amax = 0.0;
  for (int f = 0; f < 6; f++)
  {
    double a = quad_area(P[faces[f][0]], P[faces[f][1]], P[faces[f][2]], P[faces[f][3]]);
    if (a > amax)
      amax = a;
  }
  return hex_volume(P) / amax;
}

static double wave_speed(orc_model *m, long e) /* Element::getElongationWaveSpeed, Element.C:343-359 */
{
  const dnl_material *mt = &m->mat[m->emat[e]];
  double rho = 0.0;
  for (int g = 0; g < m->npe; g++)
    rho += IPV(m, DNL_IP_DENSITY, e * m->npe + g);
  rho /= m->npe;
  double nu = mt->poisson;
  return sqrt((mt->young * (1.0 - nu)) / (rho * (1.0 + nu) * (1.0 - 2.0 * nu)));
}

static double charlen(orc_model *m, long e)
{
  const int32_t *cn = m->conn + e * m->npe;
  return (m->dim == 2) ? charlen_q4(m->x, cn) : charlen_hex(m->x, cn);
}

/* Model::computeCourantTimeStep (Model.C:636-669). */
double orc_courant(orc_model *m)
{
  double crit = charlen(m, 0) / wave_speed(m, 0);
  for (long e = 1; e < m->nE; e++)
  {
    double ts = charlen(m, e) / wave_speed(m, e);
    if (ts < crit)
      crit = ts;
  }
  return crit;
}

int orc_element_lengths(orc_model *m, double *len, double *wave)
{
  for (long e = 0; e < m->nE; e++)
  {
    len[e] = charlen(m, e);
    wave[e] = wave_speed(m, e);
  }
  return DNL_OK;
}

/* Elastic stiffness matrix of one element (ElementPlane.C:182-292,
 * Element3D.C:303-399) with the Hooke matrices of Material.C:98-152
 * (axisymmetric 4x4 rr, zz, rz, tt / 3-D 6x6 xx, yy, zz, xy, yz, xz; the
 * shear terms are E/(1+nu)), on the dN/dx of the current Jacobian. */
static void stiffness(orc_model *m, long e, double *K /* [nd*nd] */)
{
  const dnl_material *mt = &m->mat[m->emat[e]];
  const double E = mt->young, nu = mt->poisson;
  const double f = E / ((1 + nu) * (1 - 2 * nu));
  int npe = m->npe, d = m->dim, nd = npe * d;
  double C[6][6] = {{0}};
  if (m->dim == 2 && m->axi)
  {
    C[0][0] = C[1][1] = C[3][3] = (1 - nu) * f;
    C[2][2] = (1 - 2 * nu) * f;
    C[1][0] = C[0][1] = C[3][0] = C[0][3] = C[3][1] = C[1][3] = nu * f;
  }
  else if (m->dim == 2)
  {
    /* Material::getHookeStiffnessMatrix(planeStrain), Material.C:105-113 */
    C[0][0] = C[1][1] = (1 - nu) * f;
    C[2][2] = (1 - 2 * nu) * f;
    C[1][0] = C[0][1] = nu * f;
  }
  else
  {
    C[0][0] = C[1][1] = C[2][2] = (1 - nu) * f;
    C[3][3] = C[4][4] = C[5][5] = (1 - 2 * nu) * f;
    C[0][1] = C[1][0] = C[0][2] = C[2][0] = C[1][2] = C[2][1] = nu * f;
  }
  memset(K, 0, sizeof(double) * nd * nd);
  double CB[6][24];
  for (int g = 0; g < npe; g++)
  {
    long q = e * npe + g;
    const double *dn = m->dNdx + q * npe * 3;
    double WxdJ = m->w[g] * m->detJ[q], R = m->radius[q];
    if (m->dim == 2)
    {
      if (m->axi)
        WxdJ *= TWO_PI * R;
      for (int i = 0; i < npe; i++)
      {
        double dNx = dn[3 * i], dNy = dn[3 * i + 1], NoR = m->axi ? m->N[g][i] / R : 0.0;
        int I = 2 * i;
        for (int r = 0; r < 4; r++)
        {
          CB[r][I] = C[r][0] * dNx + C[r][2] * dNy + C[r][3] * NoR;
          CB[r][I + 1] = C[r][1] * dNy + C[r][2] * dNx;
        }
      }
      for (int i = 0; i < npe; i++)
      {
        double dNx = dn[3 * i], dNy = dn[3 * i + 1], NoR = m->axi ? m->N[g][i] / R : 0.0;
        for (int j = 0; j < npe; j++)
        {
          int I = 2 * i, J = 2 * j;
          K[I * nd + J] += (dNx * CB[0][J] + dNy * CB[2][J]) * WxdJ;
          K[I * nd + J + 1] += (dNx * CB[0][J + 1] + dNy * CB[2][J + 1]) * WxdJ;
          K[(I + 1) * nd + J] += (dNy * CB[1][J] + dNx * CB[2][J]) * WxdJ;
          K[(I + 1) * nd + J + 1] += (dNy * CB[1][J + 1] + dNx * CB[2][J + 1]) * WxdJ;
          K[I * nd + J] += CB[3][J] * NoR * WxdJ;
          K[I * nd + J + 1] += CB[3][J + 1] * NoR * WxdJ;
        }
      }
    }
    else
    {
      for (int i = 0; i < npe; i++)
      {
        double dNx = dn[3 * i], dNy = dn[3 * i + 1], dNz = dn[3 * i + 2];
        int I = 3 * i;
        for (int r = 0; r < 6; r++)
        {
          CB[r][I] = C[r][0] * dNx + C[r][3] * dNy + C[r][5] * dNz;
          CB[r][I + 1] = C[r][1] * dNy + C[r][3] * dNx + C[r][4] * dNz;
          CB[r][I + 2] = C[r][2] * dNz + C[r][4] * dNy + C[r][5] * dNx;
        }
      }
      for (int i = 0; i < npe; i++)
      {
        double dNx = dn[3 * i], dNy = dn[3 * i + 1], dNz = dn[3 * i + 2];
        for (int j = 0; j < npe; j++)
          for (int c = 0; c < 3; c++)
          {
            int I = 3 * i, J = 3 * j + c;
            K[I * nd + J] += (dNx * CB[0][J] + dNy * CB[3][J] + dNz * CB[5][J]) * WxdJ;
            K[(I + 1) * nd + J] += (dNy * CB[1][J] + dNx * CB[3][J] + dNz * CB[4][J]) * WxdJ;
            K[(I + 2) * nd + J] += (dNz * CB[2][J] + dNy * CB[4][J] + dNx * CB[5][J]) * WxdJ;
          }
      }
    }
  }
}

/* Model::computePowerIterationTimeStep (Model.C:942-1009): the largest
 * eigenvalue of M^-1 K by power iteration, warm-started from the previous
 * vector and frequency.  As in the reference, the assembled K v is added to
 * the old vector (Vector::gatherFrom adds, Vector.C:893-915). */
static int power_iteration(orc_model *m, double *omega)
{
  int d = m->dim, npe = m->npe, nd = npe * d;
  long ndof = m->nN * d;
  if (!m->pv)
  {
    m->pv = (double *)xcalloc(ndof, sizeof(double));
    m->pv[0] = 1.0;
    for (long i = 1; i < ndof; i++)
      m->pv[i] = m->pv[i - 1] - 2. / (ndof - 1);
  }
  double *Ks = (double *)xcalloc((size_t)m->nE * nd * nd, sizeof(double));
  for (long e = 0; e < m->nE; e++)
    stiffness(m, e, Ks + (size_t)e * nd * nd);
  double *v0 = (double *)xcalloc(ndof, sizeof(double));
  double loc[24], y[24], fmax = 0.0;
  long it = 0;
  int ok = 0;
  while (!ok)
  {
    it++;
    memcpy(v0, m->pv, ndof * sizeof(double));
    for (long e = 0; e < m->nE; e++)
    {
      const int32_t *cn = m->conn + e * npe;
      for (int n = 0; n < npe; n++)
        for (int c = 0; c < d; c++)
          loc[n * d + c] = v0[cn[n] * d + c];
      const double *K = Ks + (size_t)e * nd * nd;
      for (int i = 0; i < nd; i++)
      {
        double acc = 0.0;
        for (int j = 0; j < nd; j++)
          acc += K[i * nd + j] * loc[j];
        y[i] = acc;
      }
      for (int n = 0; n < npe; n++)
        for (int c = 0; c < d; c++)
          m->pv[cn[n] * d + c] += y[n * d + c];
    }
    fmax = 0.0;
    for (long i = 0; i < ndof; i++)
    {
      m->pv[i] /= m->mass[i / d];
      if (fabs(m->pv[i]) > fmax)
        fmax = fabs(m->pv[i]);
    }
    for (long i = 0; i < ndof; i++)
      m->pv[i] /= fmax;
    double conv = fabs(fmax - m->pfmax) / fmax;
    if (conv < 1e-4)
      ok = 1;
    m->pfmax = fmax;
    if (it > 1000)
    {
      free(Ks);
      free(v0);
      m->status = DNL_ERR_POWER_ITERATION;
      return DNL_ERR_POWER_ITERATION;
    }
  }
  m->piters += it;
  free(Ks);
  free(v0);
  *omega = sqrt(fmax);
  return DNL_OK;
}

/* Solver::computeTimeStep (Solver.C:196-244). */
static int compute_time_step(orc_model *m, int force)
{
  if (force || (m->inc % m->ts_freq == 0))
  {
    double fmax;
    if (m->ts_method == DNL_TS_COURANT)
      fmax = 2.0 / orc_courant(m);
    else if (m->ts_method == DNL_TS_POWER_ITERATION)
    {
      int rc = power_iteration(m, &fmax);
      if (rc)
        return rc;
    }
    else
    {
      set_err("unknown time-step method %d", m->ts_method);
      return DNL_ERR_UNSUPPORTED;
    }
    m->dt = m->safety * m->omegaS / fmax;
  }
  return DNL_OK;
}

/* ------------------------------------------------------------ nodal update */

/* DiscreteFunction::getValue (DiscreteFunction.C:188-213), clamped at the ends. */
static double func_value(orc_model *m, int f, double t)
{
  int np = m->fnp[f];
  const double *X = m->fx[f], *Y = m->fy[f];
  if (t <= X[0])
    return Y[0];
  for (int i = 1; i < np; i++)
    if (X[i] >= t)
    {
      if (X[i] == t)
        return Y[i];
      return ((t - X[i - 1]) / (X[i] - X[i - 1])) * (Y[i] - Y[i - 1]) + Y[i - 1];
    }
  return Y[np - 1];
}

/* BoundaryCondition::applyConstantOnNewFields -> BoundaryRestrain.C:98-128 and
 * BoundarySpeed.C:139-206 for one node component. */
static void apply_bc(orc_model *m, long k, double t, double dt)
{
  int f0 = m->f0, f1 = 1 - m->f0;
  if (m->bc[k] == DNL_BC_RESTRAIN)
  {
    m->fu[f0][k] = m->fu[f1][k] = 0.0;
    m->fv[f0][k] = m->fv[f1][k] = 0.0;
    m->fa[f0][k] = m->fa[f1][k] = 0.0;
  }
  else if (m->bc[k] == DNL_BC_SPEED)
  {
    double s = m->bcv[k];
    int f = m->bcf[k];
    if (f < 0)
    {
      m->fa[f0][k] = m->fa[f1][k] = 0.0;
      m->fv[f0][k] = m->fv[f1][k] = s;
    }
    else
    {
      double a = func_value(m, f, t), b = func_value(m, f, t + dt);
      m->fa[f0][k] = (b - a) * s / dt;
      m->fa[f1][k] = m->fa[f0][k];
      m->fv[f0][k] = a * s;
      m->fv[f1][k] = b * s;
    }
    m->fu[f0][k] = m->fv[f0][k] * dt;
    m->fu[f1][k] = m->fv[f1][k] * dt;
  }
}

/* Explicit::computePredictions (Explicit.C:438-482). */
static void predictor(orc_model *m)
{
  double dt = m->dt;
  int f0 = m->f0, f1 = 1 - m->f0;
  for (long i = 0; i < m->nN; i++)
  {
    for (int c = 0; c < 3; c++)
    {
      long k = 3 * i + c;
      m->fu[f1][k] = dt * (m->fv[f0][k] + (0.5 - m->beta) * dt * m->fa[f0][k]);
      m->fv[f1][k] = m->fv[f0][k] + (1.0 - m->gamma) * dt * m->fa[f0][k];
      m->fa[f1][k] = 0.0;
    }
    for (int c = 0; c < 3; c++)
      apply_bc(m, 3 * i + c, m->t, dt);
  }
}

/* Explicit::explicitSolve (Explicit.C:489-536). */
static void corrector(orc_model *m)
{
  double dt = m->dt;
  int f0 = m->f0, f1 = 1 - m->f0, d = m->dim;
  for (long i = 0; i < m->nN; i++)
  {
    for (int c = 0; c < d; c++)
      m->fa[f1][3 * i + c] = m->fint[3 * i + c] / m->mass[i];
    for (int c = 0; c < 3; c++)
    {
      long k = 3 * i + c;
      m->fa[f1][k] -= m->alphaM * m->fa[f0][k];
      m->fa[f1][k] /= (1.0 - m->alphaM);
      m->fv[f1][k] += m->gamma * dt * m->fa[f1][k];
      m->fu[f1][k] += m->beta * (dt * dt) * m->fa[f1][k];
    }
    for (int c = 0; c < 3; c++)
      apply_bc(m, 3 * i + c, m->t, dt);
    for (int c = 0; c < 3; c++)
    {
      m->disp[3 * i + c] += m->fu[f1][3 * i + c];
      m->x[3 * i + c] += m->fu[f1][3 * i + c];
    }
  }
}

/* ------------------------------------------------------------------ driver */

/* Model::initSolve (Model.C:360-521) + Explicit.C:143-181. */
int orc_init(orc_model *m)
{
  m->status = DNL_OK;
  int rc = jacobian(m, 1);
  if (rc)
    return rc;
  mass_matrix(m);
  rc = compute_time_step(m, 1);
  if (rc)
    return rc;
  return element_pass(m, m->dt);
}

/* Increment loop of Explicit::solve (Explicit.C:184-256). */
long orc_run(orc_model *m, double t_stop, long max_incs)
{
  long k = 0;
  while (m->t < m->up_to && m->t < t_stop && (max_incs <= 0 || k < max_incs))
  {
    if (m->status)
      return -1;
    /* Explicit::updateTimes (Explicit.C:414-427) */
    if (m->t + m->dt > m->up_to)
      m->dt = m->up_to - m->t;
    m->inc++;
    predictor(m);
    if (element_pass(m, m->dt))
      return -1;
    corrector(m);
    density(m);
    /* Explicit::endStep (Explicit.C:539-552): time, then the field swap */
    m->t += m->dt;
    m->f0 = 1 - m->f0;
    if (m->t < m->up_to)
    {
      if (jacobian(m, 0))
        return -1;
      if (compute_time_step(m, 0))
        return -1;
    }
    k++;
  }
  return k;
}

/* One element pass on the current state with the given time step, followed by
 * the density update (the kernel-level parity entry point). */
int orc_element_pass(orc_model *m, double dt)
{
  int rc = jacobian(m, 0);
  if (rc)
    return rc;
  rc = element_pass(m, dt);
  if (rc)
    return rc;
  density(m);
  return DNL_OK;
}

/* sizeof of the C-ABI structs, for the ctypes layout test. */
long orc_abi_sizeof(int which)
{
  switch (which)
  {
  case 0: return (long)sizeof(dnl_model_desc);
  case 1: return (long)sizeof(dnl_material);
  case 2: return (long)sizeof(dnl_function);
  case 3: return (long)sizeof(dnl_control);
  }
  return -1;
}

void orc_control(orc_model *m, double out[4])
{
  out[0] = m->t;
  out[1] = m->dt;
  out[2] = (double)m->inc;
  out[3] = (double)m->status;
}

int orc_get_nodes(orc_model *m, int field, double *out)
{
  long n3 = 3 * m->nN;
  const double *src = NULL;
  switch (field)
  {
  case DNL_NODE_COORDS: src = m->x; break;
  case DNL_NODE_DISP: src = m->disp; break;
  case DNL_NODE_U: src = m->fu[m->f0]; break;
  case DNL_NODE_SPEED: src = m->fv[m->f0]; break;
  case DNL_NODE_ACCEL: src = m->fa[m->f0]; break;
  case DNL_NODE_SPEED_PREV: src = m->fv[1 - m->f0]; break;
  case DNL_NODE_U_PREV: src = m->fu[1 - m->f0]; break;
  case DNL_NODE_ACCEL_PREV: src = m->fa[1 - m->f0]; break;
  case DNL_NODE_FORCE: src = m->fint; break;
  case DNL_NODE_MASS:
    for (long i = 0; i < m->nN; i++)
      out[3 * i] = out[3 * i + 1] = out[3 * i + 2] = m->mass[i];
    return DNL_OK;
  default: return DNL_ERR_ARG;
  }
  memcpy(out, src, n3 * sizeof(double));
  return DNL_OK;
}

int orc_set_nodes(orc_model *m, int field, const double *in)
{
  long n3 = 3 * m->nN;
  double *dst = NULL;
  switch (field)
  {
  case DNL_NODE_COORDS: dst = m->x; break;
  case DNL_NODE_DISP: dst = m->disp; break;
  case DNL_NODE_U: dst = m->fu[m->f0]; break;
  case DNL_NODE_SPEED: dst = m->fv[m->f0]; break;
  case DNL_NODE_ACCEL: dst = m->fa[m->f0]; break;
  default: return DNL_ERR_ARG;
  }
  memcpy(dst, in, n3 * sizeof(double));
  return DNL_OK;
}

int orc_get_ips(orc_model *m, double *out)
{
  memcpy(out, m->ip, (size_t)DNL_IP_NCOMP * m->nIP * sizeof(double));
  return DNL_OK;
}

int orc_set_ips(orc_model *m, const double *in)
{
  memcpy(m->ip, in, (size_t)DNL_IP_NCOMP * m->nIP * sizeof(double));
  return DNL_OK;
}

/* Kinetic energy (Model::getTotalKineticEnergy, Model.C:612-626) and the
 * integrals of the specific internal / inelastic energies. */
int orc_energies(orc_model *m, double out[3])
{
  double ke = 0.0, ei = 0.0, ep = 0.0;
  const double *v = m->fv[m->f0];
  for (long i = 0; i < m->nN; i++)
    ke += m->mass[i] * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]) / 2.0;
  for (long e = 0; e < m->nE; e++)
  {
    const dnl_material *mt = &m->mat[m->emat[e]];
    for (int g = 0; g < m->npe; g++)
    {
      long q = e * m->npe + g;
      double wgt = mt->density * IPV(m, DNL_IP_DETJ0, q) * m->w[g] * (m->axi ? TWO_PI : 1.0);
      ei += wgt * IPV(m, DNL_IP_EINT, q);
      ep += wgt * IPV(m, DNL_IP_EINEL, q);
    }
  }
  out[0] = ke;
  out[1] = ei;
  out[2] = ep;
  return DNL_OK;
}
