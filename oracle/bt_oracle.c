/*
 * bt_oracle.c -- CPU oracle (plain C restatement) of the BlackTracer hot path.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and bench.py's
 * CPU-baseline leg as the checker.  Never linked into the product library.
 *
 * This restates, in the reference's own operation order (so that the same
 * compiler and libm give bit-identical doubles), the Kerr null-geodesic
 * integrator of BT/Metric.h, the ray set-up of BT/Grid.h:514-556, the
 * adaptive refinement of BT/Grid.h:291-505 and the T-vertex fix of
 * BT/Grid.h:103-204.  The hash maps of the reference are replaced by a dense
 * lattice; refinement decisions do not depend on set iteration order, so the
 * traced set, the values and the block levels are identical.  The T-vertex
 * fix does depend on the iteration order of the reference's unordered_map;
 * here it runs in a fixed canonical order (level ascending, then key
 * i<<32|j ascending), the order oracle/ref_harness.cpp also feeds to the
 * reference's own fixTvertices.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp).
 */
#include "bt_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* BT/Const.h:2-4 */
static const double ORC_PI = 3.141592653589793238;
#define ORC_PI2 (ORC_PI * 2.)

/* Step control constants, BT/Metric.h:27-33 */
#define ORC_SAFETY 0.9
#define ORC_PGROW -0.2
#define ORC_PSHRNK -0.25
#define ORC_ERRCON 1.89e-4
#define ORC_MAXSTP 1000
#define ORC_TINY 1.0e-30
#define ORC_ADAPTIVE 5.0

/* Cash-Karp tableau (published, Numerical Recipes); BT/Metric.h:41-49. */
static const double kb21 = 0.2, kb31 = 3.0 / 40.0, kb32 = 9.0 / 40.0,
                    kb41 = 0.3, kb42 = -0.9, kb43 = 1.2,
                    kb51 = -11.0 / 54.0, kb52 = 2.5, kb53 = -70.0 / 27.0,
                    kb54 = 35.0 / 27.0, kb61 = 1631.0 / 55296.0,
                    kb62 = 175.0 / 512.0, kb63 = 575.0 / 13824.0,
                    kb64 = 44275.0 / 110592.0, kb65 = 253.0 / 4096.0,
                    kc1 = 37.0 / 378.0, kc3 = 250.0 / 621.0,
                    kc4 = 125.0 / 594.0, kc6 = 512.0 / 1771.0,
                    kdc5 = -277.00 / 14336.0;
static const double kdc1 = 37.0 / 378.0 - 2825.0 / 27648.0,
                    kdc3 = 250.0 / 621.0 - 18575.0 / 48384.0,
                    kdc4 = 125.0 / 594.0 - 13525.0 / 55296.0,
                    kdc6 = 512.0 / 1771.0 - 0.25;

/* Newton iteration cap for the capture test.  The reference loop
 * (BT/Metric.h:152-162) has none; a ray that would spin forever there is
 * reported with status 3 here instead. */
#define ORC_NEWTON_CAP 100000

typedef struct { double a, asq; } spin_t;

static inline double sq(double x) { return x * x; }
static inline double sq3(double x) { return x * x * x; }

/* Kerr metric scalars, BT/Metric.h:64-102. */
static inline double m_delta(const spin_t* s, double r) {
  return sq(r) - 2. * r + s->asq;
}
static inline double m_sigma(const spin_t* s, double r, double th) {
  return sqrt(sq(sq(r) + s->asq) - s->asq * m_delta(s, r) * sq(sin(th)));
}
static inline double m_w(const spin_t* s, double r, double th) {
  return 2. * s->a * r / sq(m_sigma(s, r, th));
}
static inline double m_ro(const spin_t* s, double r, double th) {
  return sqrt(sq(r) + s->asq * sq(cos(th)));
}
static inline double m_rosq(const spin_t* s, double r, double th) {
  return sq(r) + s->asq * sq(cos(th));
}
static inline double m_wbar(const spin_t* s, double r, double th) {
  return m_sigma(s, r, th) * sin(th) / m_ro(s, r, th);
}
static inline double m_alpha(const spin_t* s, double r, double th) {
  return m_ro(s, r, th) * sqrt(m_delta(s, r)) / m_sigma(s, r, th);
}
static inline double m_P(const spin_t* s, double r, double b) {
  return sq(r) + s->asq - s->a * b;
}
static inline double m_R(const spin_t* s, double r, double b, double q) {
  return sq(m_P(s, r, b)) - m_delta(s, r) * (sq((b - s->a)) + q);
}
static inline double m_bigtheta(const spin_t* s, double th, double b,
                                double q) {
  return q - sq(cos(th)) * (sq(b) / sq(sin(th)) - s->asq);
}
/* BT/Metric.h:104-108 */
static inline double m_calc_speed(const spin_t* s, double r, double th) {
  double omega = 1. / (s->a + pow(r, 1.5));
  return m_wbar(s, r, th) / m_alpha(s, r, th) * (omega - m_w(s, r, th));
}

/* Camera::initforms, BT/Camera.h:54-61 */
static void cam_initforms(const spin_t* s, orc_camera* c) {
  c->alpha = m_alpha(s, c->r, c->theta);
  c->w = m_w(s, c->r, c->theta);
  c->wbar = m_wbar(s, c->r, c->theta);
  c->Delta = m_delta(s, c->r);
  c->ro = m_ro(s, c->r, c->theta);
}

void orc_camera_static(double a, double theta, double phi, double r,
                       double speed, orc_camera* c) {
  spin_t s = {a, a * a};
  memset(c, 0, sizeof(*c));
  c->theta = theta; c->phi = phi; c->r = r; c->speed = speed;
  c->bphi = 1; c->btheta = 0; c->br = 0;
  cam_initforms(&s, c);
}

void orc_camera_orbit(double a, double theta, double phi, double r, double br,
                      double btheta, double bphi, orc_camera* c) {
  spin_t s = {a, a * a};
  memset(c, 0, sizeof(*c));
  c->theta = theta; c->phi = phi; c->r = r;
  c->bphi = bphi; c->btheta = btheta; c->br = br;
  c->speed = m_calc_speed(&s, r, theta);
  cam_initforms(&s, c);
}

/* ---- capture classification, BT/Metric.h:110-174 ---- */
static double find_min_goldsec(const spin_t* s, double bval, double qval,
                               double ax, double b, double tol) {
  double gr = (sqrt(5.0) + 1.) / 2.;
  double c = b - (b - ax) / gr;
  double d = ax + (b - ax) / gr;
  while (fabs(c - d) > tol) {
    if (m_R(s, c, bval, qval) < m_R(s, d, bval, qval)) b = d;
    else ax = c;
    c = b - (b - ax) / gr;
    d = ax + (b - ax) / gr;
  }
  return (ax + b) / 2;
}
static int check_rup(const spin_t* s, double rV, double bV, double qV) {
  if (s->a == 0) return 0;
  double mn = find_min_goldsec(s, bV, qV, rV, 4 * rV, 0.00001);
  return m_R(s, mn, bV, qV) >= 0;
}
static inline double b0(const spin_t* s, double r0) {
  return -(sq3(r0) - 3. * sq(r0) + s->asq * r0 + s->asq) / (s->a * (r0 - 1.));
}
static inline double b0diff(const spin_t* s, double r0) {
  return (s->asq + s->a - 2. * r0 * (sq(r0) - 3. * r0 + 3.)) /
         (s->a * sq(r0 - 1.));
}
static inline double q0(const spin_t* s, double r0) {
  return -sq3(r0) * (sq3(r0) - 6. * sq(r0) + 9. * r0 - 4. * s->asq) /
         (s->asq * sq(r0 - 1.));
}
/* returns 1/0, or -1 when the Newton loop hits the cap */
static int check_b_q(const spin_t* s, double bV, double qV) {
  double r1 = 2. * (1. + cos(2. * acos(-s->a) / 3.));
  double r2 = 2. * (1. + cos(2. * acos(s->a) / 3.));
  double error = 0.0000001;
  double r0V = 2.0;
  double bcheck = 100;
  long it = 0;
  while (fabs(bV - bcheck) > error) {
    if (++it > ORC_NEWTON_CAP) return -1;
    bcheck = b0(s, r0V);
    double bdiffcheck = b0diff(s, r0V);
    double rnew = r0V - (bcheck - bV) / bdiffcheck;
    if (rnew < 1) r0V = 1.0001;
    else r0V = rnew;
  }
  double qb = q0(s, r0V);
  double b1 = b0(s, r2);
  double b2 = b0(s, r1);
  return (b1 >= bV) || (b2 <= bV) || (qV >= qb);
}
/* 1 = celestial (integrate), 0 = captured, -1 = Newton cap */
static int check_celest(const spin_t* s, double pRV, double rV, double bV,
                        double qV) {
  int c1 = check_b_q(s, bV, qV);
  if (c1 < 0) return -1;
  int c2 = !c1 && (pRV < 0);
  int c3 = c1 && check_rup(s, rV, bV, qV);
  return c2 || c3;
}

/* BT/Metric.h:176-185.  The phi loop is bounded (the reference's never ends
 * for -inf); identical whenever it ends within 4096 turns. */
static void wrap_to_pi(double* th, double* ph) {
  *th = fmod(*th, ORC_PI2);
  while (*th < 0) *th += ORC_PI2;
  if (*th > ORC_PI) {
    *th -= 2 * (*th - ORC_PI);
    *ph += ORC_PI;
  }
  for (int it = 0; *ph < 0; it++) {
    if (it == 4096) { *ph = fmod(*ph, ORC_PI2) + ORC_PI2; break; }
    *ph += ORC_PI2;
  }
  *ph = fmod(*ph, ORC_PI2);
}

/* Equations of motion, BT/Metric.h:198-226.  var = {r, theta, phi, pr, ptheta} */
static void derivs(const spin_t* s, const double* var, double* o, double b,
                   double q) {
  const double r = var[0], th = var[1], pr = var[3], pt = var[4];
  const double a = s->a, asq = s->asq;
  double cosv = cos(th);
  double sinv = sin(th);
  double cossq = sq(cosv);
  double sinsq = sq(sinv);
  double bsq = sq(b);
  double delta = m_delta(s, r);
  double rosq = m_rosq(s, r, th);
  double P = m_P(s, r, b);
  double prsq = sq(pr);
  double pthetasq = sq(pt);
  double R = m_R(s, r, b, q);
  double partR = (q + sq(a - b));
  double btheta = m_bigtheta(s, th, b, q);
  double rosqsq = sq(2 * rosq);
  double sqrosqdel = (sq(rosq) * delta);
  double asqcossin = asq * cosv * sinv;
  double rtwo = 2 * r - 2;

  o[0] = delta / rosq * pr;
  o[1] = 1. / rosq * pt;
  o[2] = (2 * a * P - (2 * a - 2 * b) * delta + (2 * b * cossq * delta) / sinsq) /
         (rosq * 2 * delta);
  o[3] = (rtwo * btheta - rtwo * partR + 4 * r * P) / (rosq * (2 * delta)) -
         (prsq * rtwo) / (2 * rosq) + (4 * pthetasq * r) / rosqsq -
         ((4 * r - 4) * (btheta * (delta) + R)) / (rosq * sq(2 * delta)) +
         (4 * prsq * r * (delta)) / rosqsq - (r * (btheta * delta + R)) / sqrosqdel;
  o[4] = ((2 * cosv * sinv * (bsq / sinsq - asq) +
           (2 * bsq * sq3(cosv)) / sq3(sinv)) * delta) / (rosq * 2 * delta) -
         (4 * asqcossin * pthetasq) / rosqsq -
         (4 * asqcossin * prsq * delta) / rosqsq +
         (asqcossin * (btheta * delta + R)) / sqrosqdel;
}

/* Cash-Karp step, BT/Metric.h:228-251 */
static void rkck(const spin_t* s, const double* var, const double* dvdz,
                 double h, double* out, double* err, double b, double q) {
  double aks[25], tmp[5];
  int i;
  for (i = 0; i < 5; i++) tmp[i] = var[i] + kb21 * h * dvdz[i];
  derivs(s, tmp, aks, b, q);
  for (i = 0; i < 5; i++) tmp[i] = var[i] + h * (kb31 * dvdz[i] + kb32 * aks[i]);
  derivs(s, tmp, aks + 5, b, q);
  for (i = 0; i < 5; i++)
    tmp[i] = var[i] + h * (kb41 * dvdz[i] + kb42 * aks[i] + kb43 * aks[i + 5]);
  derivs(s, tmp, aks + 10, b, q);
  for (i = 0; i < 5; i++)
    tmp[i] = var[i] + h * (kb51 * dvdz[i] + kb52 * aks[i] + kb53 * aks[i + 5] +
                           kb54 * aks[i + 10]);
  derivs(s, tmp, aks + 15, b, q);
  for (i = 0; i < 5; i++)
    tmp[i] = var[i] + h * (kb61 * dvdz[i] + kb62 * aks[i] + kb63 * aks[i + 5] +
                           kb64 * aks[i + 10] + kb65 * aks[i + 15]);
  derivs(s, tmp, aks + 20, b, q);
  for (i = 0; i < 5; i++)
    out[i] = var[i] + h * (kc1 * dvdz[i] + kc3 * aks[i + 5] + kc4 * aks[i + 10] +
                           kc6 * aks[i + 20]);
  for (i = 0; i < 5; i++)
    err[i] = h * (kdc1 * dvdz[i] + kdc3 * aks[i + 5] + kdc4 * aks[i + 10] +
                  kdc5 * aks[i + 15] + kdc6 * aks[i + 20]);
}

/* Quality-controlled step, BT/Metric.h:253-270 */
static void rkqs(const spin_t* s, double* var, const double* dvdz, double* z,
                 double* h, double eps, const double* scal, double b, double q) {
  double tmp[5], err[5];
  rkck(s, var, dvdz, *h, tmp, err, b, q);
  double errmax = 0.0;
  for (int i = 0; i < 5; i++) errmax = fmax(errmax, fabs(err[i] / scal[i]));
  errmax /= eps;
  if (errmax <= 1.0) {
    *z += *h;
    for (int i = 0; i < 5; i++) var[i] = tmp[i];
    if (errmax > ORC_ERRCON) *h = ORC_SAFETY * *h * pow(errmax, ORC_PGROW);
    else *h = ORC_ADAPTIVE * *h;
  } else {
    *h = fmin(ORC_SAFETY * *h * pow(errmax, ORC_PSHRNK), 0.1 * *h);
  }
}

static int sgnf(float v) { return (0 < v) - (v < 0); }

/* Driver, BT/Metric.h:276-303.  Returns 1 when z reached zEnd. */
static int odeint1(const spin_t* s, double* vstart, double zEnd, double eps,
                   double h1, double b, double q, int32_t maxstp,
                   int32_t* step) {
  double var[5], dvdz[5], scal[5];
  double z = 0.0;
  double h = h1 * sgnf((float)zEnd);
  for (int i = 0; i < 5; i++) var[i] = vstart[i];
  for (int nstp = 0; nstp < maxstp; nstp++) {
    derivs(s, var, dvdz, b, q);
    for (int i = 0; i < 5; i++)
      scal[i] = fabs(var[i]) + fabs(dvdz[i] * h) + ORC_TINY;
    rkqs(s, var, dvdz, &z, &h, eps, scal, b, q);
    *step = nstp;
    if (z <= zEnd) {
      for (int i = 0; i < 5; i++) vstart[i] = var[i];
      return 1;
    }
  }
  return 0;
}

/* One ray of Grid::integration_wrapper, BT/Grid.h:524-554. */
static void integrate_one(const orc_camera* cam, const spin_t* s, double th,
                          double ph, double* tho, double* pho, int32_t* st,
                          uint8_t* status, double eps, double h1, double zEnd,
                          int32_t maxstp) {
  const double thetaS = cam->theta, phiS = cam->phi, rS = cam->r;
  const double sp = cam->speed;
  double xCam = sin(th) * cos(ph);
  double yCam = sin(th) * sin(ph);
  double zCam = cos(th);

  double yFido = (-yCam + sp) / (1 - sp * yCam);
  double xFido = -sqrtf(1 - sp * sp) * xCam / (1 - sp * yCam);
  double zFido = -sqrtf(1 - sp * sp) * zCam / (1 - sp * yCam);

  double k = sqrt(1 - cam->btheta * cam->btheta);
  double rFido = xFido * cam->bphi / k + cam->br * yFido +
                 cam->br * cam->btheta / k * zFido;
  double thetaFido = cam->btheta * yFido - k * zFido;
  double phiFido = -xFido * cam->br / k + cam->bphi * yFido +
                   cam->bphi * cam->btheta / k * zFido;

  double eF = 1. / (cam->alpha + cam->w * cam->wbar * phiFido);
  double pR = eF * cam->ro * rFido / sqrtf(cam->Delta);
  double pTheta = eF * cam->ro * thetaFido;
  double pPhi = eF * cam->wbar * phiFido;

  double b = pPhi;
  double q = pTheta * pTheta +
             cos(thetaS) * cos(thetaS) * (b * b / (sin(thetaS) * sin(thetaS)) - s->asq);

  *tho = -1; *pho = -1; *st = 0; *status = 1;
  int cel = check_celest(s, pR, rS, b, q);
  if (cel < 0) { *status = 3; return; }
  if (cel) {
    double vs[5] = {rS, thetaS, phiS, pR, pTheta};
    int32_t step = 0;
    int done = odeint1(s, vs, zEnd, eps, h1, b, q, maxstp, &step);
    double to = vs[1], po = vs[2];
    wrap_to_pi(&to, &po);
    *tho = to; *pho = po; *st = step;
    *status = done ? 0 : 2;
  }
}

void orc_integrate_rays_opts(const orc_camera* cam, double a,
                             const double* theta, const double* phi, size_t n,
                             double* theta_out, double* phi_out,
                             int32_t* steps, uint8_t* status, double eps,
                             double h1, double z_end, int32_t maxstp,
                             int nthreads) {
  spin_t s = {a, a * a};
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
  for (long i = 0; i < (long)n; i++) {
    uint8_t stt;
    integrate_one(cam, &s, theta[i], phi[i], &theta_out[i], &phi_out[i],
                  &steps[i], &stt, eps, h1, z_end, maxstp);
    if (status) status[i] = stt;
  }
  (void)nthreads;
}

void orc_integrate_rays(const orc_camera* cam, double a, const double* theta,
                        const double* phi, size_t n, double* theta_out,
                        double* phi_out, int32_t* steps, uint8_t* status,
                        int nthreads) {
  /* rkckIntegrate1 constants, BT/Metric.h:311-314 */
  orc_integrate_rays_opts(cam, a, theta, phi, n, theta_out, phi_out, steps,
                          status, 1e-5, 0.01, -10000000, ORC_MAXSTP, nthreads);
}

/* ====================== adaptive grid (BT/Grid.h) ====================== */

typedef struct {
  int MAX, START, eq, N, M;
  double *th, *ph;
  uint8_t* ex;
  int32_t* steps;
  int8_t* bl;
  const orc_camera* cam;
  double a;
  int nthreads;
  long traced;
} grid_t;

void orc_grid_dims(int maxlevel, int angle, int* N, int* M) {
  int eq = angle ? 1 : 0;
  /* BT/Grid.h:612-614 */
  *N = (int)(uint32_t)round(pow(2, maxlevel) / (2 - eq) + 1);
  *M = (2 - eq) * 2 * (*N - 1);
}

/* Grid::callKernel, BT/Grid.h:382-401 (+ fillGridCam :347-355) */
static void trace_keys(grid_t* g, const uint64_t* keys, size_t n) {
  if (!n) return;
  double* th = (double*)malloc(n * sizeof(double) * 4);
  double* ph = th + n;
  double* tho = th + 2 * n;
  double* pho = th + 3 * n;
  int32_t* st = (int32_t*)malloc(n * sizeof(int32_t));
  for (size_t q = 0; q < n; q++) {
    uint32_t i = (uint32_t)(keys[q] >> 32), j = (uint32_t)keys[q];
    th[q] = (double)i / (g->N - 1) * ORC_PI / (2 - g->eq);
    ph[q] = (double)j / g->M * ORC_PI2;
  }
  orc_integrate_rays(g->cam, g->a, th, ph, n, tho, pho, st, NULL, g->nthreads);
  for (size_t q = 0; q < n; q++) {
    uint32_t i = (uint32_t)(keys[q] >> 32), j = (uint32_t)keys[q];
    size_t id = (size_t)i * g->M + j;
    g->th[id] = tho[q];
    g->ph[id] = pho[q];
    g->ex[id] = 1;
    g->steps[id] = st[q];
  }
  g->traced += (long)n;
  free(th);
  free(st);
}

typedef struct { uint64_t* v; size_t n, cap; } vec64;
static void vpush(vec64* v, uint64_t x) {
  if (v->n == v->cap) {
    v->cap = v->cap ? v->cap * 2 : 1024;
    v->v = (uint64_t*)realloc(v->v, v->cap * sizeof(uint64_t));
  }
  v->v[v->n++] = x;
}
#define KEY(i, j) (((uint64_t)(uint32_t)(i) << 32) | (uint32_t)(j))

/* Grid::refineCheck, BT/Grid.h:410-445 (disk branch disabled, :75) */
static int refine_check(grid_t* g, uint32_t i, uint32_t j, int gap, int level) {
  uint32_t k = i + gap;
  uint32_t l = (j + gap) % g->M;
  size_t M = g->M;
  double th1 = g->th[i * M + j], th2 = g->th[k * M + j];
  double th3 = g->th[i * M + l], th4 = g->th[k * M + l];
  double ph1 = g->ph[i * M + j], ph2 = g->ph[k * M + j];
  double ph3 = g->ph[i * M + l], ph4 = g->ph[k * M + l];
  double diag = (th1 - th4) * (th1 - th4) + (ph1 - ph4) * (ph1 - ph4);
  double diag2 = (th2 - th3) * (th2 - th3) + (ph2 - ph3) * (ph2 - ph3);
  double mx = diag > diag2 ? diag : diag2; /* std::max returns the first on ties */
  if (level < 6 && mx > 1E-10) return 1;
  if (mx > 0.015) return 1; /* PRECCELEST, BT/Grid.h:24 */
  g->bl[i * M + j] = (int8_t)level;
  return 0;
}

/* Grid::fillVector, BT/Grid.h:453-459: new vertices, deduplicated. */
static void fill_vector(grid_t* g, vec64* todo, uint32_t i, uint32_t j) {
  size_t id = (size_t)i * g->M + j;
  if (!g->ex[id]) {
    vpush(todo, KEY(i, j));
    g->ex[id] = 2; /* placeholder (-10,-10) until traced */
  }
}

/* --- T-vertex fix, BT/Grid.h:103-204 --- */
static int gfind(grid_t* g, uint32_t i, uint32_t j) {
  if (i >= (uint32_t)g->N || j >= (uint32_t)g->M) return 0;
  return g->ex[(size_t)i * g->M + j] != 0;
}
/* metric::check2PIcross / correct2PIcross, BT/Metric.h:333-364, factor 5 */
static void fix_2pi(double* ph, int n) {
  int cross = 0;
  for (int q = 0; q < n; q++)
    if (ph[q] > ORC_PI2 * (1. - 1. / 5.)) { cross = 1; break; }
  if (!cross) return;
  for (int q = 0; q < n; q++)
    if (ph[q] < ORC_PI2 * (1. / 5.)) ph[q] += ORC_PI2;
}
/* Grid::hermite (Paul Bourke's form, tension 0, bias 0), BT/Grid.h:183-204 */
static double hermite1(double v, double x0, double x1, double x2, double x3) {
  const double aTension = 0., aBias = 0.;
  double v2 = v * v;
  double v3 = v * v2;
  double aa = (1. + aBias) * (1. - aTension) / 2.;
  double bb = (1. - aBias) * (1. - aTension) / 2.;
  double m0 = aa * (x1 - x0) + bb * (x2 - x1);
  double m1 = aa * (x2 - x1) + bb * (x3 - x2);
  double u0 = 2. * v3 - 3. * v2 + 1.;
  double u1 = v3 - 2. * v2 + v;
  double u2 = v3 - v2;
  double u3 = -2. * v3 + 3. * v2;
  return u0 * x1 + u1 * m0 + u2 * m1 + u3 * x2;
}

static void check_adjacent(grid_t* g, uint64_t ij, uint64_t ij2, int level,
                           int udlr, int gap) {
  const uint32_t M = (uint32_t)g->M, N = (uint32_t)g->N;
  uint32_t i0 = (uint32_t)(ij >> 32), j0 = (uint32_t)ij;
  uint32_t i = i0 + udlr * gap / 2;
  uint32_t j = j0 + (1 - udlr) * gap / 2;
  if (!gfind(g, i, j)) return;
  uint32_t jprev = (j0 - (1 - udlr) * gap + M) % M;
  uint32_t jnext = (j0 + (1 - udlr) * 2 * gap) % M;
  uint32_t iprev = i0 - udlr * gap;
  uint32_t inext = i0 + 2 * udlr * gap;
  int half = 0;
  if (i0 == 0) {
    jprev = (j0 + M / 2) % M;
    iprev = gap;
  } else if (inext > N - 1) {
    inext = i0;
    if (g->eq) jnext = (j0 + M / 2) % M;
    else half = 1;
  }
  uint32_t i2 = (uint32_t)(ij2 >> 32), j2 = (uint32_t)ij2;
  size_t id = (size_t)i * M + j;
  size_t idA = (size_t)i0 * M + j0, idB = (size_t)i2 * M + j2;
  int succes = 0;
  if (gfind(g, iprev, jprev) && gfind(g, inext, jnext)) {
    size_t idP = (size_t)iprev * M + jprev, idN = (size_t)inext * M + jnext;
    double ct[4] = {g->th[idP], g->th[idA], g->th[idB], g->th[idN]};
    double cp[4] = {g->ph[idP], g->ph[idA], g->ph[idB], g->ph[idN]};
    int prevnul = (ct[0] == -1 && cp[0] == -1);
    int nextnul = (ct[3] == -1 && cp[3] == -1);
    if (!prevnul && !nextnul) {
      succes = 1;
      if (half) ct[3] = ORC_PI - ct[3];
      fix_2pi(cp, 4);
      g->th[id] = hermite1(0.5, ct[0], ct[1], ct[2], ct[3]);
      g->ph[id] = hermite1(0.5, cp[0], cp[1], cp[2], cp[3]);
    }
  }
  if (!succes) {
    double ct[2] = {g->th[idA], g->th[idB]};
    double cp[2] = {g->ph[idA], g->ph[idB]};
    fix_2pi(cp, 2);
    g->th[id] = 1. / 2. * (ct[1] + ct[0]);
    g->ph[id] = 1. / 2. * (cp[1] + cp[0]);
  }
  if (level + 1 == g->MAX) return;
  check_adjacent(g, ij, KEY(i, j), level + 1, udlr, gap / 2);
  check_adjacent(g, KEY(i, j), ij2, level + 1, udlr, gap / 2);
}

/* Grid::fixTvertices, BT/Grid.h:103-119 */
static void fix_tvertices(grid_t* g, uint32_t i, uint32_t j, int level) {
  if (level == g->MAX) return;
  if (g->ph[(size_t)i * g->M + j] < 0) return;
  int gap = (int)pow(2, g->MAX - level);
  uint32_t k = i + gap;
  uint32_t l = (j + gap) % g->M;
  check_adjacent(g, KEY(i, j), KEY(k, j), level, 1, gap);
  check_adjacent(g, KEY(i, j), KEY(i, l), level, 0, gap);
  check_adjacent(g, KEY(i, l), KEY(k, l), level, 1, gap);
  check_adjacent(g, KEY(k, j), KEY(k, l), level, 0, gap);
}

long orc_grid_build(int maxlevel, int startlevel, int angle,
                    const orc_camera* cam, double a, int tfix_order,
                    double* theta, double* phi, uint8_t* exists,
                    int32_t* steps, int8_t* blevel, int nthreads) {
  if (maxlevel < startlevel || startlevel < 1 || maxlevel > 14) return -1;
  grid_t g;
  memset(&g, 0, sizeof(g));
  g.MAX = maxlevel; g.START = startlevel; g.eq = angle ? 1 : 0;
  orc_grid_dims(maxlevel, angle, &g.N, &g.M);
  g.th = theta; g.ph = phi; g.ex = exists; g.steps = steps; g.bl = blevel;
  g.cam = cam; g.a = a; g.nthreads = nthreads;
  const size_t NM = (size_t)g.N * g.M;
  for (size_t q = 0; q < NM; q++) { theta[q] = -2; phi[q] = -2; }
  memset(exists, 0, NM);
  memset(steps, 0, NM * sizeof(int32_t));
  memset(blevel, -1, NM);
  const uint32_t N = (uint32_t)g.N, M = (uint32_t)g.M;

  /* raytrace, BT/Grid.h:291-319 */
  int gap = (int)pow(2, g.MAX - g.START);
  vec64 start = {0}, check = {0}, todo = {0}, toint = {0};
  vpush(&start, 0);
  if (g.eq) vpush(&start, KEY(N - 1, 0));
  trace_keys(&g, start.v, start.n);
  for (uint32_t j = 0; j < M; j += gap) {
    size_t id = j;
    g.th[id] = g.th[0]; g.ph[id] = g.ph[0]; g.ex[id] = 1;
    g.steps[id] = g.steps[0];
    vpush(&check, KEY(0, j));
    if (g.eq) {
      size_t s0 = (size_t)(N - 1) * M;
      id = s0 + j;
      g.th[id] = g.th[s0]; g.ph[id] = g.ph[s0]; g.ex[id] = 1;
      g.steps[id] = g.steps[0]; /* the reference copies steps[0] (:312) */
    }
  }
  /* integrateFirst, BT/Grid.h:325-338 */
  for (uint32_t i = gap; i < N - g.eq; i += gap) {
    for (uint32_t j = 0; j < M; j += gap) {
      vpush(&toint, KEY(i, j));
      if (i == N - 1) ;
      else if (g.MAX == g.START) g.bl[(size_t)i * M + j] = (int8_t)g.START;
      else vpush(&check, KEY(i, j));
    }
  }
  trace_keys(&g, toint.v, toint.n);

  /* adaptiveBlockIntegration, BT/Grid.h:465-505 */
  int level = g.START;
  int early = 0;
  while (level < g.MAX) {
    if (check.n == 0) { early = 1; break; }
    todo.n = 0; toint.n = 0;
    uint32_t bgap = (uint32_t)pow(2, g.MAX - level);
    for (size_t q = 0; q < check.n; q++) {
      uint32_t i = (uint32_t)(check.v[q] >> 32), j = (uint32_t)check.v[q];
      uint32_t k = i + bgap / 2;
      uint32_t l = j + bgap / 2;
      j = j % M;
      if (refine_check(&g, i, j, bgap, level)) {
        fill_vector(&g, &toint, k, j);
        fill_vector(&g, &toint, k, l);
        fill_vector(&g, &toint, i, l);
        fill_vector(&g, &toint, i + bgap, l);
        fill_vector(&g, &toint, k, (j + bgap) % M);
        vpush(&todo, KEY(i, j));
        vpush(&todo, KEY(k, j));
        vpush(&todo, KEY(k, l));
        vpush(&todo, KEY(i, l));
      }
    }
    trace_keys(&g, toint.v, toint.n);
    level++;
    vec64 t = check; check = todo; todo = t;
  }
  if (!early)
    for (size_t q = 0; q < check.n; q++) {
      uint32_t i = (uint32_t)(check.v[q] >> 32), j = (uint32_t)check.v[q];
      g.bl[(size_t)i * M + j] = (int8_t)level;
    }

  /* T-vertex fix in canonical order (level, then key), BT/Grid.h:620-622 */
  if (tfix_order == 1) {
    for (int lv = g.START; lv < g.MAX; lv++)
      for (uint32_t i = 0; i < N; i++)
        for (uint32_t j = 0; j < M; j++)
          if (g.bl[(size_t)i * M + j] == lv) fix_tvertices(&g, i, j, lv);
  }
  for (size_t q = 0; q < NM; q++)
    if (exists[q] != 1) { exists[q] = 0; }
  free(start.v); free(check.v); free(todo.v); free(toint.v);
  return g.traced;
}
