/* FP64 direct summation, the accuracy oracle for every FMM result.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/ and bench.py to measure the error
 * of FMM outputs against the exact sum.  Restates kernel_apply /
 * kernel_apply_single_check (flexmm/flexmm2d/helpers.py:91-116): the sum over
 * all sources, skipping a source that coincides with the target in both
 * coordinates when `check` is set.
 *
 * Build: gcc -O2 -fopenmp -shared -fPIC direct.c -o _build/liboracle_direct.so -lm
 * (no -ffast-math: the sums are plain IEEE double).
 */
#include <math.h>
#include <stdint.h>

/* Laplace: -log(|t-s|^2) / (4 pi), examples/kifmm_laplace.py:24-29 */
void oracle_direct_laplace(const double *sx, const double *sy, const double *tau,
                           int64_t ns, const double *tx, const double *ty,
                           int64_t nt, int check, double *out)
{
    const double c = 1.0 / (4.0 * M_PI);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t j = 0; j < nt; ++j) {
        double acc = 0.0;
        const double x = tx[j], y = ty[j];
        for (int64_t i = 0; i < ns; ++i) {
            double dx = x - sx[i], dy = y - sy[i];
            if (check && dx == 0.0 && dy == 0.0) continue;
            acc += -log(dx * dx + dy * dy) * c * tau[i];
        }
        out[j] = acc;
    }
}

/* Laplace potential and its gradient in the target position, rows
 * out[0..2][nt] = (u, du/dx, du/dy): the reference's Gradient_Eval
 * (examples/pure_kifmm_laplace_gradient.py:32-55) summed over all sources,
 * with the same coincidence skip (flexmm/kifmm2d/scalar/helpers.py:200-205). */
void oracle_direct_laplace_grad(const double *sx, const double *sy, const double *tau,
                                int64_t ns, const double *tx, const double *ty,
                                int64_t nt, int check, double *out)
{
    const double c = 1.0 / (4.0 * M_PI), g = -1.0 / (2.0 * M_PI);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t j = 0; j < nt; ++j) {
        double u = 0.0, ux = 0.0, uy = 0.0;
        const double x = tx[j], y = ty[j];
        for (int64_t i = 0; i < ns; ++i) {
            double dx = x - sx[i], dy = y - sy[i];
            if (check && dx == 0.0 && dy == 0.0) continue;
            double d2 = dx * dx + dy * dy;
            u += -log(d2) * c * tau[i];
            ux += g * dx / d2 * tau[i];
            uy += g * dy / d2 * tau[i];
        }
        out[j] = u;
        out[nt + j] = ux;
        out[2 * nt + j] = uy;
    }
}

/* Stokeslet direct sum: rows out[0..2][nt] = (u, v, p) from forces (fx, fy),
 * kernel_apply_single / kernel_apply_single_check of
 * flexmm/kifmm2d/vector/stokes_fmm.py:100-187: u, v scaled by 1/(4 pi),
 * p by 1/(2 pi); coincident pairs skipped when check. */
void oracle_direct_stokes(const double *sx, const double *sy, const double *fx,
                          const double *fy, int64_t ns, const double *tx, const double *ty,
                          int64_t nt, int check, double *out)
{
    const double us = 0.25 / M_PI, ps = 0.5 / M_PI;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t j = 0; j < nt; ++j) {
        double u = 0.0, v = 0.0, p = 0.0;
        const double x = tx[j], y = ty[j];
        for (int64_t i = 0; i < ns; ++i) {
            double dx = x - sx[i], dy = y - sy[i];
            if (check && dx == 0.0 && dy == 0.0) continue;
            double id2 = 1.0 / (dx * dx + dy * dy);
            double logid = 0.5 * log(id2);
            double dxdy = dx * dy * id2;
            u += (logid + dx * dx * id2) * fx[i] + dxdy * fy[i];
            v += dxdy * fx[i] + (logid + dy * dy * id2) * fy[i];
            p += (fx[i] * dx + fy[i] * dy) * id2;
        }
        out[j] = u * us;
        out[nt + j] = v * us;
        out[2 * nt + j] = p * ps;
    }
}

/* Laplace single plus double layer: the reference example's
 * Laplace_Both_Eval (examples/pure_kifmm_laplace_dipoles.py:31-40),
 *   -log(d^2)/(4 pi) slp + (n . d)/d^2 / (2 pi) dlp,  d = target - source,
 * summed over all sources (normal (nx, ny) per source), coincident pairs
 * skipped when check (flexmm/kifmm2d/scalar/helpers.py:200-205). */
void oracle_direct_laplace_dipole(const double *sx, const double *sy, const double *slp,
                                  const double *dlp, const double *nx, const double *ny,
                                  int64_t ns, const double *tx, const double *ty, int64_t nt,
                                  int check, double *out)
{
    const double c = 1.0 / (4.0 * M_PI), g = 1.0 / (2.0 * M_PI);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t j = 0; j < nt; ++j) {
        double acc = 0.0;
        const double x = tx[j], y = ty[j];
        for (int64_t i = 0; i < ns; ++i) {
            double dx = x - sx[i], dy = y - sy[i];
            if (check && dx == 0.0 && dy == 0.0) continue;
            double d2 = dx * dx + dy * dy;
            acc += -log(d2) * c * slp[i] + (nx[i] * dx + ny[i] * dy) / d2 * g * dlp[i];
        }
        out[j] = acc;
    }
}

/* Stokeslets plus stresslets: the reference's
 * kernel_apply_single(_check)_with_dipole (flexmm/kifmm2d/vector/stokes_fmm.py:
 * 128-235) summed over all sources: forces (fx, fy), double-layer strengths
 * (sx_, sy_) along the normals (nx, ny); rows (u, v, p). */
void oracle_direct_stokes_dipole(const double *sx, const double *sy, const double *fx,
                                 const double *fy, const double *gx, const double *gy,
                                 const double *nx, const double *ny, int64_t ns,
                                 const double *tx, const double *ty, int64_t nt, int check,
                                 double *out)
{
    const double us = 0.25 / M_PI, ps = 0.5 / M_PI;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t j = 0; j < nt; ++j) {
        double u = 0.0, v = 0.0, p = 0.0;
        const double x = tx[j], y = ty[j];
        for (int64_t i = 0; i < ns; ++i) {
            double dx = x - sx[i], dy = y - sy[i];
            if (check && dx == 0.0 && dy == 0.0) continue;
            double id2 = 1.0 / (dx * dx + dy * dy);
            double logid = 0.5 * log(id2);
            double dxdy = dx * dy * id2;
            double dn = dx * nx[i] + dy * ny[i];
            double c = 4.0 * dn * id2 * id2;
            u += (logid + dx * dx * id2) * fx[i] + dxdy * fy[i] + c * dx * dx * gx[i] + c * dx * dy * gy[i];
            v += dxdy * fx[i] + (logid + dy * dy * id2) * fy[i] + c * dx * dy * gx[i] + c * dy * dy * gy[i];
            p += (fx[i] * dx + fy[i] * dy) * id2;
            p += 2.0 * (-nx[i] * id2 + 0.5 * dx * c) * gx[i] + 2.0 * (-ny[i] * id2 + 0.5 * dy * c) * gy[i];
        }
        out[j] = u * us;
        out[nt + j] = v * us;
        out[2 * nt + j] = p * ps;
    }
}
