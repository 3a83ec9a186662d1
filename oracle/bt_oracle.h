/*
 * bt_oracle.h -- CPU oracle for the BlackTracer hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (annemiekie/BlackTracer), used by tests/, the smoke check and the
 * CPU-baseline leg of bench.py as the thing results are CHECKED against.  The
 * product library (blacktracer_b200/) never links, loads or calls it.
 *
 * Every function cites the reference file:line it restates.  Paths are
 * relative to the reference project root; "BT/" = BlackTracer2/BlackTracer/.
 *
 * Parity of this restatement is pinned against the reference's own code,
 * compiled in place from the reference sources into oracle/_ref/ by
 * oracle/Makefile (see oracle/ref_harness.cpp); tests/test_oracle_pin.py and
 * the committed fixtures in tests/golden/ hold that pin.
 */
#ifndef BT_ORACLE_H
#define BT_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Field-for-field copy of the reference Camera (BT/Camera.h:8-11). */
typedef struct orc_camera {
  double theta, phi, r;
  double speed, br, btheta, bphi;
  double alpha, w, wbar, Delta, ro;
} orc_camera;

/* Camera(theta, phi, r, speed): BT/Camera.h:27-38 (static / custom speed). */
void orc_camera_static(double a, double theta, double phi, double r,
                       double speed, orc_camera* out);
/* Camera(theta, phi, r, br, btheta, bphi): BT/Camera.h:40-52 (Keplerian). */
void orc_camera_orbit(double a, double theta, double phi, double r, double br,
                      double btheta, double bphi, orc_camera* out);

/* Grid::integration_wrapper, BT/Grid.h:514-556, for n rays.  Captured rays
 * give (-1, -1, 0).  Ray status (0 escaped-and-integrated, 1 captured,
 * 2 MAXSTP reached, 3 capture-test Newton did not converge within the cap). */
void orc_integrate_rays(const orc_camera* cam, double a, const double* theta,
                        const double* phi, size_t n, double* theta_out,
                        double* phi_out, int32_t* steps, uint8_t* status,
                        int nthreads);

/* Integration with non-default tolerance / end point / cap (BT/Metric.h:276
 * odeint1 called directly, as the relative-tolerance variant of the C1
 * configuration uses). */
void orc_integrate_rays_opts(const orc_camera* cam, double a,
                             const double* theta, const double* phi, size_t n,
                             double* theta_out, double* phi_out,
                             int32_t* steps, uint8_t* status, double eps,
                             double h1, double z_end, int32_t maxstp,
                             int nthreads);

/* Adaptive grid, BT/Grid.h:605-624, on a dense N x M lattice.
 *   tfix_order: 0 = no T-vertex fix (raw traced values),
 *               1 = T-vertex fix in canonical order: blocks sorted by
 *                   (level ascending, key = i<<32|j ascending).
 * Outputs (caller-allocated, N*M each, row-major i*M+j):
 *   theta/phi  : vertex values, -2 where no vertex exists
 *   exists     : 1 where a vertex exists (CamToCel has the key)
 *   steps      : the reference's steps vector (BT/Grid.h:577)
 *   blevel     : level of the leaf block whose top-left corner is (i,j), or -1
 * Returns the number of rays traced, or -1 on bad arguments. */
long orc_grid_build(int maxlevel, int startlevel, int angle,
                    const orc_camera* cam, double a, int tfix_order,
                    double* theta, double* phi, uint8_t* exists,
                    int32_t* steps, int8_t* blevel, int nthreads);
void orc_grid_dims(int maxlevel, int angle, int* N, int* M);

#ifdef __cplusplus
}
#endif
#endif
