/*
 * clover_oracle.c -- CPU restatement of the CloverLeaf hydro path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  See
 * clover_oracle.h for the conventions.  Each function names the reference
 * routine it restates as file:line (paths inside the CloverLeaf project).
 * Build without FMA contraction (-ffp-contract=off) so the arithmetic is the
 * reference serial build's arithmetic bit for bit.
 */
#include "clover_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define G_SMALL 1.0e-16 /* driver/definitions.h:34 */
#define G_BIG 1.0e+21   /* driver/definitions.h:35 */

#define AT(a, i, j) (a)[(size_t)(j) * (size_t)sx + (size_t)(i)]

oc_chunk *oc_create(int nx, int ny, double gamma) {
  if (nx < 1 || ny < 1) return NULL;
  oc_chunk *c = (oc_chunk *)calloc(1, sizeof(oc_chunk));
  if (!c) return NULL;
  c->nx = nx;
  c->ny = ny;
  c->sx = nx + 5;
  c->sy = ny + 5;
  c->gamma = gamma;
  size_t n2 = (size_t)c->sx * (size_t)c->sy;
  size_t n1 = (size_t)((nx > ny ? nx : ny) + 6);
  for (int f = 0; f < OC_NUM_2D; ++f) {
    c->f[f] = (double *)calloc(n2, sizeof(double));
    if (!c->f[f]) { oc_destroy(c); return NULL; }
  }
  for (int g = 0; g < OC_NUM_1D; ++g) {
    c->g[g] = (double *)calloc(n1, sizeof(double));
    if (!c->g[g]) { oc_destroy(c); return NULL; }
  }
  return c;
}

void oc_destroy(oc_chunk *c) {
  if (!c) return;
  for (int f = 0; f < OC_NUM_2D; ++f) free(c->f[f]);
  for (int g = 0; g < OC_NUM_1D; ++g) free(c->g[g]);
  free(c);
}

size_t oc_index(const oc_chunk *c, int i, int j) { return (size_t)j * (size_t)c->sx + (size_t)i; }
double *oc_field(oc_chunk *c, int id) { return (id >= 0 && id < OC_NUM_2D) ? c->f[id] : NULL; }
double *oc_geom(oc_chunk *c, int id) { return (id >= 0 && id < OC_NUM_1D) ? c->g[id] : NULL; }

/* src/serial/build_field.cpp:29-180 -- every array starts at zero. */
void oc_build_field(oc_chunk *c) {
  size_t n2 = (size_t)c->sx * (size_t)c->sy;
  size_t n1 = (size_t)((c->nx > c->ny ? c->nx : c->ny) + 6);
  for (int f = 0; f < OC_NUM_2D; ++f) memset(c->f[f], 0, n2 * sizeof(double));
  for (int g = 0; g < OC_NUM_1D; ++g) memset(c->g[g], 0, n1 * sizeof(double));
}

/* src/serial/initialise_chunk.cpp:30-85 (single tile, t_left = t_bottom = 1). */
void oc_initialise_chunk(oc_chunk *c, double gxmin, double gymin, double gxmax, double gymax) {
  const int sx = c->sx;
  const int x_min = 1, y_min = 1, x_max = c->nx, y_max = c->ny;
  double dx = (gxmax - gxmin) / (double)(c->nx);
  double dy = (gymax - gymin) / (double)(c->ny);
  double xmin = gxmin + dx * (double)(1 - 1);
  double ymin = gymin + dy * (double)(1 - 1);
  double *vertexx = c->g[OC_VERTEXX], *vertexdx = c->g[OC_VERTEXDX];
  double *vertexy = c->g[OC_VERTEXY], *vertexdy = c->g[OC_VERTEXDY];
  double *cellx = c->g[OC_CELLX], *celldx = c->g[OC_CELLDX];
  double *celly = c->g[OC_CELLY], *celldy = c->g[OC_CELLDY];
  const int xrange = (x_max + 3) - (x_min - 2) + 1;
  const int yrange = (y_max + 3) - (y_min - 2) + 1;
  for (int j = 0; j < xrange; j++) {
    vertexx[j] = xmin + dx * (j - 1 - x_min);
    vertexdx[j] = dx;
  }
  for (int k = 0; k < yrange; k++) {
    vertexy[k] = ymin + dy * (k - 1 - y_min);
    vertexdy[k] = dy;
  }
  const int xrange1 = (x_max + 2) - (x_min - 2) + 1;
  const int yrange1 = (y_max + 2) - (y_min - 2) + 1;
  for (int j = 0; j < xrange1; j++) {
    cellx[j] = 0.5 * (vertexx[j] + vertexx[j + 1]);
    celldx[j] = dx;
  }
  for (int k = 0; k < yrange1; k++) {
    celly[k] = 0.5 * (vertexy[k] + vertexy[k + 1]);
    celldy[k] = dy;
  }
  double *volume = c->f[OC_VOLUME], *xarea = c->f[OC_XAREA], *yarea = c->f[OC_YAREA];
  for (int j = 0; j < yrange1; j++) {
    for (int i = 0; i < xrange1; i++) {
      AT(volume, i, j) = dx * dy;
      AT(xarea, i, j) = celldy[j];
      AT(yarea, i, j) = celldx[i];
    }
  }
}

/* src/serial/generate_chunk.cpp:31-131.  State 0 is the background. */
void oc_generate_chunk(oc_chunk *c, int nstates, const oc_state *st) {
  const int sx = c->sx;
  const int xrange = (c->nx + 2) - (1 - 2) + 1;
  const int yrange = (c->ny + 2) - (1 - 2) + 1;
  double *e0 = c->f[OC_ENERGY0], *d0 = c->f[OC_DENSITY0];
  double *u0 = c->f[OC_XVEL0], *v0 = c->f[OC_YVEL0];
  const double *vertexx = c->g[OC_VERTEXX], *vertexy = c->g[OC_VERTEXY];
  const double *cellx = c->g[OC_CELLX], *celly = c->g[OC_CELLY];
  for (int j = 0; j < yrange; j++) {
    for (int i = 0; i < xrange; i++) {
      AT(e0, i, j) = st[0].energy;
      AT(d0, i, j) = st[0].density;
      AT(u0, i, j) = st[0].xvel;
      AT(v0, i, j) = st[0].yvel;
    }
  }
  for (int s = 1; s < nstates; ++s) {
    for (int j = 0; j < yrange; j++) {
      for (int i = 0; i < xrange; i++) {
        double x_cent = st[s].xmin;
        double y_cent = st[s].ymin;
        int hit = 0;
        if (st[s].geometry == 1) {
          hit = (vertexx[i + 1] >= st[s].xmin && vertexx[i] < st[s].xmax) &&
                (vertexy[j + 1] >= st[s].ymin && vertexy[j] < st[s].ymax);
        } else if (st[s].geometry == 2) {
          double radius = sqrt((cellx[i] - x_cent) * (cellx[i] - x_cent) + (celly[j] - y_cent) * (celly[j] - y_cent));
          hit = radius <= st[s].radius;
        } else if (st[s].geometry == 3) {
          hit = vertexx[i] == x_cent && vertexy[j] == y_cent;
        }
        if (hit) {
          AT(e0, i, j) = st[s].energy;
          AT(d0, i, j) = st[s].density;
          for (int kt = j; kt <= j + 1; ++kt) {
            for (int jt = i; jt <= i + 1; ++jt) {
              AT(u0, jt, kt) = st[s].xvel;
              AT(v0, jt, kt) = st[s].yvel;
            }
          }
        }
      }
    }
  }
}

/* src/serial/ideal_gas.cpp:28-48 (gamma generalised) and :55-66. */
void oc_ideal_gas(oc_chunk *c, int predict) {
  const int sx = c->sx;
  const double *density = c->f[predict ? OC_DENSITY1 : OC_DENSITY0];
  const double *energy = c->f[predict ? OC_ENERGY1 : OC_ENERGY0];
  double *pressure = c->f[OC_PRESSURE], *soundspeed = c->f[OC_SOUNDSPEED];
  const double gm1 = c->gamma - 1.0;
  for (int j = 2; j < c->ny + 2; j++) {
    for (int i = 2; i < c->nx + 2; i++) {
      double v = 1.0 / AT(density, i, j);
      AT(pressure, i, j) = gm1 * AT(density, i, j) * AT(energy, i, j);
      double pressurebyenergy = gm1 * AT(density, i, j);
      double pressurebyvolume = -AT(density, i, j) * AT(pressure, i, j);
      double sound_speed_squared = v * v * (AT(pressure, i, j) * pressurebyenergy - pressurebyvolume);
      AT(soundspeed, i, j) = sqrt(sound_speed_squared);
    }
  }
}

/* src/serial/viscosity.cpp:30-68, including the diry-tests-pgradx quirk (:57). */
void oc_viscosity(oc_chunk *c) {
  const int sx = c->sx;
  const double *celldx = c->g[OC_CELLDX], *celldy = c->g[OC_CELLDY];
  const double *density0 = c->f[OC_DENSITY0], *pressure = c->f[OC_PRESSURE];
  const double *xvel0 = c->f[OC_XVEL0], *yvel0 = c->f[OC_YVEL0];
  double *viscosity = c->f[OC_VISCOSITY];
  for (int j = 2; j < c->ny + 2; j++) {
    for (int i = 2; i < c->nx + 2; i++) {
      double ugrad = (AT(xvel0, i + 1, j) + AT(xvel0, i + 1, j + 1)) - (AT(xvel0, i, j) + AT(xvel0, i, j + 1));
      double vgrad = (AT(yvel0, i, j + 1) + AT(yvel0, i + 1, j + 1)) - (AT(yvel0, i, j) + AT(yvel0, i + 1, j));
      double div = (celldx[i] * (ugrad) + celldy[j] * (vgrad));
      double strain2 = 0.5 * (AT(xvel0, i, j + 1) + AT(xvel0, i + 1, j + 1) - AT(xvel0, i, j) - AT(xvel0, i + 1, j)) / celldy[j] +
                       0.5 * (AT(yvel0, i + 1, j) + AT(yvel0, i + 1, j + 1) - AT(yvel0, i, j) - AT(yvel0, i, j + 1)) / celldx[i];
      double pgradx = (AT(pressure, i + 1, j) - AT(pressure, i - 1, j)) / (celldx[i] + celldx[i + 1]);
      double pgrady = (AT(pressure, i, j + 1) - AT(pressure, i, j - 1)) / (celldy[j] + celldy[j + 2]);
      double pgradx2 = pgradx * pgradx;
      double pgrady2 = pgrady * pgrady;
      double limiter = ((0.5 * (ugrad) / celldx[i]) * pgradx2 + (0.5 * (vgrad) / celldy[j]) * pgrady2 + strain2 * pgradx * pgrady) /
                       fmax(pgradx2 + pgrady2, G_SMALL);
      if ((limiter > 0.0) || (div >= 0.0)) {
        AT(viscosity, i, j) = 0.0;
      } else {
        double dirx = 1.0;
        if (pgradx < 0.0) dirx = -1.0;
        pgradx = dirx * fmax(G_SMALL, fabs(pgradx));
        double diry = 1.0;
        if (pgradx < 0.0) diry = -1.0;
        pgrady = diry * fmax(G_SMALL, fabs(pgrady));
        double pgrad = sqrt(pgradx * pgradx + pgrady * pgrady);
        double xgrad = fabs(celldx[i] * pgrad / pgradx);
        double ygrad = fabs(celldy[j] * pgrad / pgrady);
        double grad = fmin(xgrad, ygrad);
        double grad2 = grad * grad;
        AT(viscosity, i, j) = 2.0 * AT(density0, i, j) * grad2 * limiter * limiter;
      }
    }
  }
}

/* src/serial/calc_dt.cpp:30-111 (the diagnostic print of :85-110 is left to
 * the caller; control is always 1 = "sound"). */
double oc_calc_dt(oc_chunk *c, double dtmin, double dtc_safe, double dtu_safe, double dtv_safe,
                  double dtdiv_safe, int *control, int *jldt, int *kldt, int *small) {
  const int sx = c->sx;
  const double *celldx = c->g[OC_CELLDX], *celldy = c->g[OC_CELLDY];
  const double *xarea = c->f[OC_XAREA], *yarea = c->f[OC_YAREA], *volume = c->f[OC_VOLUME];
  const double *density0 = c->f[OC_DENSITY0], *viscosity_a = c->f[OC_VISCOSITY];
  const double *soundspeed = c->f[OC_SOUNDSPEED], *xvel0 = c->f[OC_XVEL0], *yvel0 = c->f[OC_YVEL0];
  double dt_min_val = G_BIG;
  double jk_control = 1.1;
  double dt_min_val0 = dt_min_val;
  for (int j = 2; j < c->ny + 2; j++) {
    for (int i = 2; i < c->nx + 2; i++) {
      double dsx = celldx[i];
      double dsy = celldy[j];
      double cc = AT(soundspeed, i, j) * AT(soundspeed, i, j);
      cc = cc + 2.0 * AT(viscosity_a, i, j) / AT(density0, i, j);
      cc = fmax(sqrt(cc), G_SMALL);
      double dtct = dtc_safe * fmin(dsx, dsy) / cc;
      double div = 0.0;
      double dv1 = (AT(xvel0, i, j) + AT(xvel0, i, j + 1)) * AT(xarea, i, j);
      double dv2 = (AT(xvel0, i + 1, j) + AT(xvel0, i + 1, j + 1)) * AT(xarea, i + 1, j);
      div = div + dv2 - dv1;
      double dtut = dtu_safe * 2.0 * AT(volume, i, j) / fmax(fmax(fabs(dv1), fabs(dv2)), G_SMALL * AT(volume, i, j));
      dv1 = (AT(yvel0, i, j) + AT(yvel0, i + 1, j)) * AT(yarea, i, j);
      dv2 = (AT(yvel0, i, j + 1) + AT(yvel0, i + 1, j + 1)) * AT(yarea, i, j + 1);
      div = div + dv2 - dv1;
      double dtvt = dtv_safe * 2.0 * AT(volume, i, j) / fmax(fmax(fabs(dv1), fabs(dv2)), G_SMALL * AT(volume, i, j));
      div = div / (2.0 * AT(volume, i, j));
      double dtdivt;
      if (div < -G_SMALL) {
        dtdivt = dtdiv_safe * (-1.0 / div);
      } else {
        dtdivt = G_BIG;
      }
      double mins = fmin(dtct, fmin(dtut, fmin(dtvt, fmin(dtdivt, G_BIG))));
      dt_min_val0 = fmin(mins, dt_min_val0);
    }
  }
  dt_min_val = dt_min_val0;
  *control = (int)(10.01 * (jk_control - (int)(jk_control)));
  jk_control = jk_control - (jk_control - (int)(jk_control));
  *jldt = ((int)jk_control) % c->nx;
  *kldt = (int)(1.f + (jk_control / c->nx));
  *small = dt_min_val < dtmin ? 1 : 0;
  return dt_min_val;
}

/* src/serial/PdV.cpp:36-87. */
void oc_pdv_kernel(oc_chunk *c, int predict, double dt) {
  const int sx = c->sx;
  const double *xarea = c->f[OC_XAREA], *yarea = c->f[OC_YAREA], *volume = c->f[OC_VOLUME];
  const double *density0 = c->f[OC_DENSITY0], *energy0 = c->f[OC_ENERGY0];
  const double *pressure = c->f[OC_PRESSURE], *viscosity = c->f[OC_VISCOSITY];
  const double *xvel0 = c->f[OC_XVEL0], *yvel0 = c->f[OC_YVEL0];
  const double *xvel1 = c->f[OC_XVEL1], *yvel1 = c->f[OC_YVEL1];
  double *density1 = c->f[OC_DENSITY1], *energy1 = c->f[OC_ENERGY1];
  for (int j = 2; j < c->ny + 2; j++) {
    for (int i = 2; i < c->nx + 2; i++) {
      double left_flux, right_flux, bottom_flux, top_flux;
      if (predict) {
        left_flux = (AT(xarea, i, j) * (AT(xvel0, i, j) + AT(xvel0, i, j + 1) + AT(xvel0, i, j) + AT(xvel0, i, j + 1))) * 0.25 * dt * 0.5;
        right_flux = (AT(xarea, i + 1, j) * (AT(xvel0, i + 1, j) + AT(xvel0, i + 1, j + 1) + AT(xvel0, i + 1, j) + AT(xvel0, i + 1, j + 1))) *
                     0.25 * dt * 0.5;
        bottom_flux = (AT(yarea, i, j) * (AT(yvel0, i, j) + AT(yvel0, i + 1, j) + AT(yvel0, i, j) + AT(yvel0, i + 1, j))) * 0.25 * dt * 0.5;
        top_flux = (AT(yarea, i, j + 1) * (AT(yvel0, i, j + 1) + AT(yvel0, i + 1, j + 1) + AT(yvel0, i, j + 1) + AT(yvel0, i + 1, j + 1))) *
                   0.25 * dt * 0.5;
      } else {
        left_flux = (AT(xarea, i, j) * (AT(xvel0, i, j) + AT(xvel0, i, j + 1) + AT(xvel1, i, j) + AT(xvel1, i, j + 1))) * 0.25 * dt;
        right_flux = (AT(xarea, i + 1, j) * (AT(xvel0, i + 1, j) + AT(xvel0, i + 1, j + 1) + AT(xvel1, i + 1, j) + AT(xvel1, i + 1, j + 1))) *
                     0.25 * dt;
        bottom_flux = (AT(yarea, i, j) * (AT(yvel0, i, j) + AT(yvel0, i + 1, j) + AT(yvel1, i, j) + AT(yvel1, i + 1, j))) * 0.25 * dt;
        top_flux = (AT(yarea, i, j + 1) * (AT(yvel0, i, j + 1) + AT(yvel0, i + 1, j + 1) + AT(yvel1, i, j + 1) + AT(yvel1, i + 1, j + 1))) *
                   0.25 * dt;
      }
      double total_flux = right_flux - left_flux + top_flux - bottom_flux;
      double volume_change_s = AT(volume, i, j) / (AT(volume, i, j) + total_flux);
      double recip_volume = 1.0 / AT(volume, i, j);
      double energy_change = (AT(pressure, i, j) / AT(density0, i, j) + AT(viscosity, i, j) / AT(density0, i, j)) * total_flux * recip_volume;
      AT(energy1, i, j) = AT(energy0, i, j) - energy_change;
      AT(density1, i, j) = AT(density0, i, j) * volume_change_s;
    }
  }
}

/* src/serial/revert.cpp:29-41. */
void oc_revert(oc_chunk *c) {
  const int sx = c->sx;
  for (int j = 2; j < c->ny + 2; j++) {
    for (int i = 2; i < c->nx + 2; i++) {
      AT(c->f[OC_DENSITY1], i, j) = AT(c->f[OC_DENSITY0], i, j);
      AT(c->f[OC_ENERGY1], i, j) = AT(c->f[OC_ENERGY0], i, j);
    }
  }
}

/* src/serial/accelerate.cpp:28-56. */
void oc_accelerate(oc_chunk *c, double dt) {
  const int sx = c->sx;
  const double *xarea = c->f[OC_XAREA], *yarea = c->f[OC_YAREA], *volume = c->f[OC_VOLUME];
  const double *density0 = c->f[OC_DENSITY0], *pressure = c->f[OC_PRESSURE], *viscosity = c->f[OC_VISCOSITY];
  const double *xvel0 = c->f[OC_XVEL0], *yvel0 = c->f[OC_YVEL0];
  double *xvel1 = c->f[OC_XVEL1], *yvel1 = c->f[OC_YVEL1];
  double halfdt = 0.5 * dt;
  for (int j = 2; j < c->ny + 3; j++) {
    for (int i = 2; i < c->nx + 3; i++) {
      double stepbymass_s = halfdt / ((AT(density0, i - 1, j - 1) * AT(volume, i - 1, j - 1) + AT(density0, i - 1, j) * AT(volume, i - 1, j) +
                                       AT(density0, i, j) * AT(volume, i, j) + AT(density0, i, j - 1) * AT(volume, i, j - 1)) *
                                      0.25);
      AT(xvel1, i, j) = AT(xvel0, i, j) - stepbymass_s * (AT(xarea, i, j) * (AT(pressure, i, j) - AT(pressure, i - 1, j)) +
                                                          AT(xarea, i, j - 1) * (AT(pressure, i, j - 1) - AT(pressure, i - 1, j - 1)));
      AT(yvel1, i, j) = AT(yvel0, i, j) - stepbymass_s * (AT(yarea, i, j) * (AT(pressure, i, j) - AT(pressure, i, j - 1)) +
                                                          AT(yarea, i - 1, j) * (AT(pressure, i - 1, j) - AT(pressure, i - 1, j - 1)));
      AT(xvel1, i, j) = AT(xvel1, i, j) - stepbymass_s * (AT(xarea, i, j) * (AT(viscosity, i, j) - AT(viscosity, i - 1, j)) +
                                                          AT(xarea, i, j - 1) * (AT(viscosity, i, j - 1) - AT(viscosity, i - 1, j - 1)));
      AT(yvel1, i, j) = AT(yvel1, i, j) - stepbymass_s * (AT(yarea, i, j) * (AT(viscosity, i, j) - AT(viscosity, i, j - 1)) +
                                                          AT(yarea, i - 1, j) * (AT(viscosity, i - 1, j) - AT(viscosity, i - 1, j - 1)));
    }
  }
}

/* src/serial/flux_calc.cpp:27-43. */
void oc_flux_calc(oc_chunk *c, double dt) {
  const int sx = c->sx;
  const double *xarea = c->f[OC_XAREA], *yarea = c->f[OC_YAREA];
  const double *xvel0 = c->f[OC_XVEL0], *yvel0 = c->f[OC_YVEL0];
  const double *xvel1 = c->f[OC_XVEL1], *yvel1 = c->f[OC_YVEL1];
  double *vol_flux_x = c->f[OC_VOL_FLUX_X], *vol_flux_y = c->f[OC_VOL_FLUX_Y];
  for (int j = 2; j < c->ny + 3; j++) {
    for (int i = 2; i < c->nx + 3; i++) {
      AT(vol_flux_x, i, j) = 0.25 * dt * AT(xarea, i, j) * (AT(xvel0, i, j) + AT(xvel0, i, j + 1) + AT(xvel1, i, j) + AT(xvel1, i, j + 1));
      AT(vol_flux_y, i, j) = 0.25 * dt * AT(yarea, i, j) * (AT(yvel0, i, j) + AT(yvel0, i + 1, j) + AT(yvel1, i, j) + AT(yvel1, i + 1, j));
    }
  }
}

/* The van Leer limited donor value used twice per face in
 * src/serial/advec_cell.cpp:84-112 (and :176-204). */
static inline double cell_limiter(double sigma, double sigma3, double sigma4, double diffuw, double diffdw) {
  const double one_by_six = 1.0 / 6.0;
  double wind = 1.0;
  if (diffdw <= 0.0) wind = -1.0;
  if (diffuw * diffdw > 0.0) {
    return (1.0 - sigma) * wind * fmin(fmin(fabs(diffuw), fabs(diffdw)), one_by_six * (sigma3 * fabs(diffuw) + sigma4 * fabs(diffdw)));
  }
  return 0.0;
}

/* src/serial/advec_cell.cpp:28-220 with the work arrays of :229-231. */
void oc_advec_cell(oc_chunk *c, int sweep_number, int dir) {
  const int sx = c->sx;
  const int x_max = c->nx, y_max = c->ny;
  const double *vertexdx = c->g[OC_VERTEXDX], *vertexdy = c->g[OC_VERTEXDY];
  const double *volume = c->f[OC_VOLUME];
  double *density1 = c->f[OC_DENSITY1], *energy1 = c->f[OC_ENERGY1];
  double *mass_flux_x = c->f[OC_MASS_FLUX_X], *mass_flux_y = c->f[OC_MASS_FLUX_Y];
  const double *vol_flux_x = c->f[OC_VOL_FLUX_X], *vol_flux_y = c->f[OC_VOL_FLUX_Y];
  double *pre_vol = c->f[OC_WORK1], *post_vol = c->f[OC_WORK2];
  double *ener_flux = c->f[OC_WORK7];
  if (dir == 1) {
    for (int j = 0; j < y_max + 4; j++) {
      for (int i = 0; i < x_max + 4; i++) {
        if (sweep_number == 1) {
          AT(pre_vol, i, j) = AT(volume, i, j) + (AT(vol_flux_x, i + 1, j) - AT(vol_flux_x, i, j) + AT(vol_flux_y, i, j + 1) - AT(vol_flux_y, i, j));
          AT(post_vol, i, j) = AT(pre_vol, i, j) - (AT(vol_flux_x, i + 1, j) - AT(vol_flux_x, i, j));
        } else {
          AT(pre_vol, i, j) = AT(volume, i, j) + AT(vol_flux_x, i + 1, j) - AT(vol_flux_x, i, j);
          AT(post_vol, i, j) = AT(volume, i, j);
        }
      }
    }
    for (int j = 2; j < y_max + 2; j++) {
      for (int i = 2; i < x_max + 4; i++) {
        int upwind, donor, downwind, dif;
        if (AT(vol_flux_x, i, j) > 0.0) {
          upwind = i - 2; donor = i - 1; downwind = i; dif = donor;
        } else {
          upwind = (i + 1 < x_max + 2) ? i + 1 : x_max + 2;
          donor = i; downwind = i - 1; dif = upwind;
        }
        double sigmat = fabs(AT(vol_flux_x, i, j)) / AT(pre_vol, donor, j);
        double sigma3 = (1.0 + sigmat) * (vertexdx[i] / vertexdx[dif]);
        double sigma4 = 2.0 - sigmat;
        double sigmav = sigmat;
        double limiter = cell_limiter(sigmav, sigma3, sigma4, AT(density1, donor, j) - AT(density1, upwind, j),
                                      AT(density1, downwind, j) - AT(density1, donor, j));
        AT(mass_flux_x, i, j) = AT(vol_flux_x, i, j) * (AT(density1, donor, j) + limiter);
        double sigmam = fabs(AT(mass_flux_x, i, j)) / (AT(density1, donor, j) * AT(pre_vol, donor, j));
        limiter = cell_limiter(sigmam, sigma3, sigma4, AT(energy1, donor, j) - AT(energy1, upwind, j),
                               AT(energy1, downwind, j) - AT(energy1, donor, j));
        AT(ener_flux, i, j) = AT(mass_flux_x, i, j) * (AT(energy1, donor, j) + limiter);
      }
    }
    for (int j = 2; j < y_max + 2; j++) {
      for (int i = 2; i < x_max + 2; i++) {
        double pre_mass_s = AT(density1, i, j) * AT(pre_vol, i, j);
        double post_mass_s = pre_mass_s + AT(mass_flux_x, i, j) - AT(mass_flux_x, i + 1, j);
        double post_ener_s = (AT(energy1, i, j) * pre_mass_s + AT(ener_flux, i, j) - AT(ener_flux, i + 1, j)) / post_mass_s;
        double advec_vol_s = AT(pre_vol, i, j) + AT(vol_flux_x, i, j) - AT(vol_flux_x, i + 1, j);
        AT(density1, i, j) = post_mass_s / advec_vol_s;
        AT(energy1, i, j) = post_ener_s;
      }
    }
  } else if (dir == 2) {
    for (int j = 0; j < y_max + 4; j++) {
      for (int i = 0; i < x_max + 4; i++) {
        if (sweep_number == 1) {
          AT(pre_vol, i, j) = AT(volume, i, j) + (AT(vol_flux_y, i, j + 1) - AT(vol_flux_y, i, j) + AT(vol_flux_x, i + 1, j) - AT(vol_flux_x, i, j));
          AT(post_vol, i, j) = AT(pre_vol, i, j) - (AT(vol_flux_y, i, j + 1) - AT(vol_flux_y, i, j));
        } else {
          AT(pre_vol, i, j) = AT(volume, i, j) + AT(vol_flux_y, i, j + 1) - AT(vol_flux_y, i, j);
          AT(post_vol, i, j) = AT(volume, i, j);
        }
      }
    }
    for (int j = 2; j < y_max + 4; j++) {
      for (int i = 2; i < x_max + 2; i++) {
        int upwind, donor, downwind, dif;
        if (AT(vol_flux_y, i, j) > 0.0) {
          upwind = j - 2; donor = j - 1; downwind = j; dif = donor;
        } else {
          upwind = (j + 1 < y_max + 2) ? j + 1 : y_max + 2;
          donor = j; downwind = j - 1; dif = upwind;
        }
        double sigmat = fabs(AT(vol_flux_y, i, j)) / AT(pre_vol, i, donor);
        double sigma3 = (1.0 + sigmat) * (vertexdy[j] / vertexdy[dif]);
        double sigma4 = 2.0 - sigmat;
        double sigmav = sigmat;
        double limiter = cell_limiter(sigmav, sigma3, sigma4, AT(density1, i, donor) - AT(density1, i, upwind),
                                      AT(density1, i, downwind) - AT(density1, i, donor));
        AT(mass_flux_y, i, j) = AT(vol_flux_y, i, j) * (AT(density1, i, donor) + limiter);
        double sigmam = fabs(AT(mass_flux_y, i, j)) / (AT(density1, i, donor) * AT(pre_vol, i, donor));
        limiter = cell_limiter(sigmam, sigma3, sigma4, AT(energy1, i, donor) - AT(energy1, i, upwind),
                               AT(energy1, i, downwind) - AT(energy1, i, donor));
        AT(ener_flux, i, j) = AT(mass_flux_y, i, j) * (AT(energy1, i, donor) + limiter);
      }
    }
    for (int j = 2; j < y_max + 2; j++) {
      for (int i = 2; i < x_max + 2; i++) {
        double pre_mass_s = AT(density1, i, j) * AT(pre_vol, i, j);
        double post_mass_s = pre_mass_s + AT(mass_flux_y, i, j) - AT(mass_flux_y, i, j + 1);
        double post_ener_s = (AT(energy1, i, j) * pre_mass_s + AT(ener_flux, i, j) - AT(ener_flux, i, j + 1)) / post_mass_s;
        double advec_vol_s = AT(pre_vol, i, j) + AT(vol_flux_y, i, j) - AT(vol_flux_y, i, j + 1);
        AT(density1, i, j) = post_mass_s / advec_vol_s;
        AT(energy1, i, j) = post_ener_s;
      }
    }
  }
}

/* The limited nodal velocity flux of src/serial/advec_mom.cpp:118-131 (x) and
 * :190-203 (y). */
static inline double mom_limited(double vdiffuw, double vdiffdw, double sigma, double width, double dx_dif) {
  double limiter = 0.0;
  if (vdiffuw * vdiffdw > 0.0) {
    double auw = fabs(vdiffuw);
    double adw = fabs(vdiffdw);
    double wind = 1.0;
    if (vdiffdw <= 0.0) wind = -1.0;
    limiter = wind * fmin(fmin(width * ((2.0 - sigma) * adw / width + (1.0 + sigma) * auw / dx_dif) / 6.0, auw), adw);
  }
  return limiter;
}

/* src/serial/advec_mom.cpp:30-225 with the work arrays of :233-242. */
void oc_advec_mom(oc_chunk *c, int which_vel, int sweep_number, int direction) {
  const int sx = c->sx;
  const int x_max = c->nx, y_max = c->ny;
  double *vel1 = c->f[which_vel == 1 ? OC_XVEL1 : OC_YVEL1];
  const double *mass_flux_x = c->f[OC_MASS_FLUX_X], *mass_flux_y = c->f[OC_MASS_FLUX_Y];
  const double *vol_flux_x = c->f[OC_VOL_FLUX_X], *vol_flux_y = c->f[OC_VOL_FLUX_Y];
  const double *volume = c->f[OC_VOLUME], *density1 = c->f[OC_DENSITY1];
  const double *celldx = c->g[OC_CELLDX], *celldy = c->g[OC_CELLDY];
  double *node_flux = c->f[OC_WORK1], *node_mass_post = c->f[OC_WORK2], *node_mass_pre = c->f[OC_WORK3];
  double *mom_flux = c->f[OC_WORK4], *pre_vol = c->f[OC_WORK5], *post_vol = c->f[OC_WORK6];
  int mom_sweep = direction + 2 * (sweep_number - 1);
  for (int j = 0; j < y_max + 4; j++) {
    for (int i = 0; i < x_max + 4; i++) {
      if (mom_sweep == 1) {
        AT(post_vol, i, j) = AT(volume, i, j) + AT(vol_flux_y, i, j + 1) - AT(vol_flux_y, i, j);
        AT(pre_vol, i, j) = AT(post_vol, i, j) + AT(vol_flux_x, i + 1, j) - AT(vol_flux_x, i, j);
      } else if (mom_sweep == 2) {
        AT(post_vol, i, j) = AT(volume, i, j) + AT(vol_flux_x, i + 1, j) - AT(vol_flux_x, i, j);
        AT(pre_vol, i, j) = AT(post_vol, i, j) + AT(vol_flux_y, i, j + 1) - AT(vol_flux_y, i, j);
      } else if (mom_sweep == 3) {
        AT(post_vol, i, j) = AT(volume, i, j);
        AT(pre_vol, i, j) = AT(post_vol, i, j) + AT(vol_flux_y, i, j + 1) - AT(vol_flux_y, i, j);
      } else if (mom_sweep == 4) {
        AT(post_vol, i, j) = AT(volume, i, j);
        AT(pre_vol, i, j) = AT(post_vol, i, j) + AT(vol_flux_x, i + 1, j) - AT(vol_flux_x, i, j);
      }
    }
  }
  if (direction == 1) {
    if (which_vel == 1) {
      for (int j = 2; j < y_max + 3; j++) {
        for (int i = 0; i < x_max + 4; i++) {
          AT(node_flux, i, j) = 0.25 * (AT(mass_flux_x, i, j - 1) + AT(mass_flux_x, i, j) + AT(mass_flux_x, i + 1, j - 1) + AT(mass_flux_x, i + 1, j));
        }
      }
      for (int j = 2; j < y_max + 3; j++) {
        for (int i = 1; i < x_max + 4; i++) {
          AT(node_mass_post, i, j) = 0.25 * (AT(density1, i, j - 1) * AT(post_vol, i, j - 1) + AT(density1, i, j) * AT(post_vol, i, j) +
                                             AT(density1, i - 1, j - 1) * AT(post_vol, i - 1, j - 1) + AT(density1, i - 1, j) * AT(post_vol, i - 1, j));
          AT(node_mass_pre, i, j) = AT(node_mass_post, i, j) - AT(node_flux, i - 1, j) + AT(node_flux, i, j);
        }
      }
    }
    for (int j = 2; j < y_max + 3; j++) {
      for (int i = 1; i < x_max + 3; i++) {
        int upwind, donor, downwind, dif;
        if (AT(node_flux, i, j) < 0.0) {
          upwind = i + 2; donor = i + 1; downwind = i; dif = donor;
        } else {
          upwind = i - 1; donor = i; downwind = i + 1; dif = upwind;
        }
        double sigma = fabs(AT(node_flux, i, j)) / (AT(node_mass_pre, donor, j));
        double width = celldx[i];
        double vdiffuw = AT(vel1, donor, j) - AT(vel1, upwind, j);
        double vdiffdw = AT(vel1, downwind, j) - AT(vel1, donor, j);
        double limiter = mom_limited(vdiffuw, vdiffdw, sigma, width, celldx[dif]);
        double advec_vel_s = AT(vel1, donor, j) + (1.0 - sigma) * limiter;
        AT(mom_flux, i, j) = advec_vel_s * AT(node_flux, i, j);
      }
    }
    for (int j = 2; j < y_max + 3; j++) {
      for (int i = 2; i < x_max + 3; i++) {
        AT(vel1, i, j) = (AT(vel1, i, j) * AT(node_mass_pre, i, j) + AT(mom_flux, i - 1, j) - AT(mom_flux, i, j)) / AT(node_mass_post, i, j);
      }
    }
  } else if (direction == 2) {
    if (which_vel == 1) {
      for (int j = 0; j < y_max + 4; j++) {
        for (int i = 2; i < x_max + 3; i++) {
          AT(node_flux, i, j) = 0.25 * (AT(mass_flux_y, i - 1, j) + AT(mass_flux_y, i, j) + AT(mass_flux_y, i - 1, j + 1) + AT(mass_flux_y, i, j + 1));
        }
      }
      for (int j = 1; j < y_max + 4; j++) {
        for (int i = 2; i < x_max + 3; i++) {
          AT(node_mass_post, i, j) = 0.25 * (AT(density1, i, j - 1) * AT(post_vol, i, j - 1) + AT(density1, i, j) * AT(post_vol, i, j) +
                                             AT(density1, i - 1, j - 1) * AT(post_vol, i - 1, j - 1) + AT(density1, i - 1, j) * AT(post_vol, i - 1, j));
          AT(node_mass_pre, i, j) = AT(node_mass_post, i, j) - AT(node_flux, i, j - 1) + AT(node_flux, i, j);
        }
      }
    }
    for (int j = 1; j < y_max + 3; j++) {
      for (int i = 2; i < x_max + 3; i++) {
        int upwind, donor, downwind, dif;
        if (AT(node_flux, i, j) < 0.0) {
          upwind = j + 2; donor = j + 1; downwind = j; dif = donor;
        } else {
          upwind = j - 1; donor = j; downwind = j + 1; dif = upwind;
        }
        double sigma = fabs(AT(node_flux, i, j)) / (AT(node_mass_pre, i, donor));
        double width = celldy[j];
        double vdiffuw = AT(vel1, i, donor) - AT(vel1, i, upwind);
        double vdiffdw = AT(vel1, i, downwind) - AT(vel1, i, donor);
        double limiter = mom_limited(vdiffuw, vdiffdw, sigma, width, celldy[dif]);
        double advec_vel_s = AT(vel1, i, donor) + (1.0 - sigma) * limiter;
        AT(mom_flux, i, j) = advec_vel_s * AT(node_flux, i, j);
      }
    }
    for (int j = 2; j < y_max + 3; j++) {
      for (int i = 2; i < x_max + 3; i++) {
        AT(vel1, i, j) = (AT(vel1, i, j) * AT(node_mass_pre, i, j) + AT(mom_flux, i, j - 1) - AT(mom_flux, i, j)) / AT(node_mass_post, i, j);
      }
    }
  }
}

/* src/serial/reset_field.cpp:28-51. */
void oc_reset_field(oc_chunk *c) {
  const int sx = c->sx;
  for (int j = 2; j < c->ny + 2; j++) {
    for (int i = 2; i < c->nx + 2; i++) {
      AT(c->f[OC_DENSITY0], i, j) = AT(c->f[OC_DENSITY1], i, j);
      AT(c->f[OC_ENERGY0], i, j) = AT(c->f[OC_ENERGY1], i, j);
    }
  }
  for (int j = 2; j < c->ny + 3; j++) {
    for (int i = 2; i < c->nx + 3; i++) {
      AT(c->f[OC_XVEL0], i, j) = AT(c->f[OC_XVEL1], i, j);
      AT(c->f[OC_YVEL0], i, j) = AT(c->f[OC_YVEL1], i, j);
    }
  }
}

/*
 * src/serial/update_halo.cpp:33-684.  Each field class has its own source
 * rows/columns and sign flips; the table below restates them, quirks included:
 *   cell fields:   bottom (j,1-k) <- (j,2+k); top (j,ny+2+k) <- (j,ny+1-k);
 *                  left (1-j,k) <- (2+j,k); right (nx+2+j,k) <- (nx+1-j,k);
 *                  soundspeed's bottom reads (j,k) instead of (j,2+k) (:273).
 *   vertex fields: bottom (j,1-k) <- (j,3+k); top (j,ny+3+k) <- (j,ny+1-k);
 *                  left (1-j,k) <- (3+j,k); right (nx+3+j,k) <- (nx+1-j,k);
 *                  xvel flips sign on left/right, yvel on bottom/top.
 *   x-face fields: bottom (j,1-k) <- (j,3+k); top (j,ny+2+k) <- (j,ny-k);
 *                  left (1-j,k) <- -(3+j,k); right (nx+3+j,k) <- -(nx+1-j,k).
 *   y-face fields: bottom (j,1-k) <- -(j,3+k); top (j,ny+3+k) <- -(j,ny+1-k);
 *                  left (1-j,k) <- (3+j,k); right (nx+2+j,k) <- (nx-j,k).
 * Bottom/top run first over the whole row (halo columns included), then
 * left/right over the whole column, so corners end up from the left/right pass.
 */
typedef struct {
  int xe, ye;               /* extra extent over the cell range: 1 for node/face dims */
  int bot_src, top_dst, top_src, left_src, right_dst, right_src;
  double sign_bt, sign_lr;
  int soundspeed_quirk;
} halo_rule;

static halo_rule rule_for(int field) {
  halo_rule r;
  memset(&r, 0, sizeof r);
  switch (field) {
    case OC_XVEL0: case OC_XVEL1: case OC_YVEL0: case OC_YVEL1:
      r.xe = 1; r.ye = 1; r.bot_src = 3; r.top_dst = 3; r.top_src = 1; r.left_src = 3; r.right_dst = 3; r.right_src = 1;
      r.sign_bt = (field == OC_YVEL0 || field == OC_YVEL1) ? -1.0 : 1.0;
      r.sign_lr = (field == OC_XVEL0 || field == OC_XVEL1) ? -1.0 : 1.0;
      break;
    case OC_VOL_FLUX_X: case OC_MASS_FLUX_X:
      r.xe = 1; r.ye = 0; r.bot_src = 3; r.top_dst = 2; r.top_src = 0; r.left_src = 3; r.right_dst = 3; r.right_src = 1;
      r.sign_bt = 1.0; r.sign_lr = -1.0;
      break;
    case OC_VOL_FLUX_Y: case OC_MASS_FLUX_Y:
      r.xe = 0; r.ye = 1; r.bot_src = 3; r.top_dst = 3; r.top_src = 1; r.left_src = 3; r.right_dst = 2; r.right_src = 0;
      r.sign_bt = -1.0; r.sign_lr = 1.0;
      break;
    default: /* cell data */
      r.xe = 0; r.ye = 0; r.bot_src = 2; r.top_dst = 2; r.top_src = 1; r.left_src = 2; r.right_dst = 2; r.right_src = 1;
      r.sign_bt = 1.0; r.sign_lr = 1.0;
      r.soundspeed_quirk = field == OC_SOUNDSPEED;
      break;
  }
  return r;
}

void oc_update_halo(oc_chunk *c, const int fields[15], int depth) { oc_update_halo_faces(c, fields, depth, 15); }

/* The same fill on the faces in `faces` only (bits 1 left, 2 right, 4 bottom,
 * 8 top): update_halo_kernel fills a face when the chunk's and the tile's
 * neighbours on it are both external (src/serial/update_halo.cpp:41-71). */
void oc_update_halo_faces(oc_chunk *c, const int fields[15], int depth, int faces) {
  const int sx = c->sx;
  const int x_max = c->nx, y_max = c->ny;
  for (int f = 0; f < 15; ++f) {
    if (fields[f] != 1) continue;
    halo_rule r = rule_for(f);
    double *a = c->f[f];
    /* bottom then top over j in [x_min - depth, x_max + xe + depth] (C: 2-depth .. x_max+1+xe+depth) */
    if (faces & 4)
      for (int j = 2 - depth; j < x_max + r.xe + depth + 2; j++) {
        for (int k = 0; k < depth; ++k) {
          int src = r.soundspeed_quirk ? k : r.bot_src + k;
          AT(a, j, 1 - k) = r.sign_bt * AT(a, j, src);
        }
      }
    if (faces & 8)
      for (int j = 2 - depth; j < x_max + r.xe + depth + 2; j++) {
        for (int k = 0; k < depth; ++k) {
          AT(a, j, y_max + r.top_dst + k) = r.sign_bt * AT(a, j, y_max + r.top_src - k);
        }
      }
    if (faces & 1)
      for (int k = 2 - depth; k < y_max + r.ye + depth + 2; k++) {
        for (int j = 0; j < depth; ++j) {
          AT(a, 1 - j, k) = r.sign_lr * AT(a, r.left_src + j, k);
        }
      }
    if (faces & 2)
      for (int k = 2 - depth; k < y_max + r.ye + depth + 2; k++) {
        for (int j = 0; j < depth; ++j) {
          AT(a, x_max + r.right_dst + j, k) = r.sign_lr * AT(a, x_max + r.right_src - j, k);
        }
      }
  }
}

/* One of update_tile_halo_{l,r,b,t}_kernel (src/serial/update_tile_halo_kernel.cpp,
 * called from driver/update_tile_halo.cpp:27-91): dst's halo on `side` (1 left,
 * 2 right, 4 bottom, 8 top) from src, the tile on that side, for the listed
 * fields, `depth` deep.  Tile-local indices (x_min = y_min = 1, C index = that
 * + 1).  Along the strip the loops run over [x_min - depth, x_max + depth]
 * (one further for nodes, and for the faces that extend that way: y faces on
 * a left/right strip, x faces on a bottom/top one -- the rule's ye / xe);
 * across it, the halo element k of dst takes src's k-th interior element from
 * the shared face, one further in for nodes and the faces normal to the strip
 * on the right and top sides (the rule's xe / ye). */
void oc_tile_halo(oc_chunk *dst, const oc_chunk *src, int side, const int fields[15], int depth) {
  const size_t dsx = (size_t)dst->sx, ssx = (size_t)src->sx;
  for (int f = 0; f < 15; ++f) {
    if (fields[f] != 1) continue;
    const halo_rule r = rule_for(f);
    double *d = dst->f[f];
    const double *s = src->f[f];
    if (side == 1 || side == 2) {
      for (int k = 2 - depth; k < dst->ny + r.ye + depth + 2; k++) {
        for (int j = 0; j < depth; ++j) {
          if (side == 1) /* left: density0(x_min - j, k) = left_density0(left_xmax + 1 - j, k) */
            d[(size_t)k * dsx + (size_t)(1 - j)] = s[(size_t)k * ssx + (size_t)(src->nx + 1 - j)];
          else /* right: density0(x_max + 2 + j, k) = right_density0(right_xmin - 1 + 2 + j, k); +1 for xvel / x faces */
            d[(size_t)k * dsx + (size_t)(dst->nx + 2 + r.xe + j)] = s[(size_t)k * ssx + (size_t)(2 + r.xe + j)];
        }
      }
    } else {
      for (int k = 0; k < depth; ++k) {
        for (int j = 2 - depth; j < dst->nx + r.xe + depth + 2; j++) {
          if (side == 4) /* bottom: density0(j, y_min - k) = bottom_density0(j, bottom_ymax + 1 - k) */
            d[(size_t)(1 - k) * dsx + (size_t)j] = s[(size_t)(src->ny + 1 - k) * ssx + (size_t)j];
          else /* top: density0(j, y_max + 2 + k) = top_density0(j, top_ymin - 1 + 2 + k); +1 for yvel / y faces */
            d[(size_t)(dst->ny + 2 + r.ye + k) * dsx + (size_t)j] = s[(size_t)(2 + r.ye + k) * ssx + (size_t)j];
        }
      }
    }
  }
}

/* src/serial/field_summary.cpp:44-104 (ideal_gas first, then the sums in the
 * reference's sequential order). */
void oc_field_summary(oc_chunk *c, double out[5]) {
  const int sx = c->sx;
  oc_ideal_gas(c, 0);
  const double *xvel0 = c->f[OC_XVEL0], *yvel0 = c->f[OC_YVEL0], *volume = c->f[OC_VOLUME];
  const double *density0 = c->f[OC_DENSITY0], *energy0 = c->f[OC_ENERGY0], *pressure = c->f[OC_PRESSURE];
  double vol = 0.0, mass = 0.0, ie = 0.0, ke = 0.0, press = 0.0;
  const int nx = c->nx, ny = c->ny;
  for (int idx = 0; idx < ny * nx; idx++) {
    const int j = 2 + idx % nx;
    const int k = 2 + idx / nx;
    double vsqrd = 0.0;
    for (int kv = k; kv <= k + 1; ++kv) {
      for (int jv = j; jv <= j + 1; ++jv) {
        vsqrd += 0.25 * (AT(xvel0, jv, kv) * AT(xvel0, jv, kv) + AT(yvel0, jv, kv) * AT(yvel0, jv, kv));
      }
    }
    double cell_vol = AT(volume, j, k);
    double cell_mass = cell_vol * AT(density0, j, k);
    vol += cell_vol;
    mass += cell_mass;
    ie += cell_mass * AT(energy0, j, k);
    ke += cell_mass * 0.5 * vsqrd;
    press += cell_vol * AT(pressure, j, k);
  }
  out[0] = vol; out[1] = mass; out[2] = ie; out[3] = ke; out[4] = press;
}

/* Double-double accumulation (Knuth two-sum), so the result is the per-cell
 * terms summed with ~1e-30 relative error whatever the order. */
typedef struct { double hi, lo; } dd;
static inline void dd_add(dd *s, double x) {
  double t = s->hi + x;
  double bp = t - s->hi;
  double err = (s->hi - (t - bp)) + (x - bp);
  s->hi = t;
  s->lo += err;
}

void oc_field_summary_exact(oc_chunk *c, double out[5]) {
  const int sx = c->sx;
  oc_ideal_gas(c, 0);
  const double *xvel0 = c->f[OC_XVEL0], *yvel0 = c->f[OC_YVEL0], *volume = c->f[OC_VOLUME];
  const double *density0 = c->f[OC_DENSITY0], *energy0 = c->f[OC_ENERGY0], *pressure = c->f[OC_PRESSURE];
  dd s[5] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}};
  for (int k = 2; k < c->ny + 2; k++) {
    for (int j = 2; j < c->nx + 2; j++) {
      double vsqrd = 0.0;
      for (int kv = k; kv <= k + 1; ++kv)
        for (int jv = j; jv <= j + 1; ++jv)
          vsqrd += 0.25 * (AT(xvel0, jv, kv) * AT(xvel0, jv, kv) + AT(yvel0, jv, kv) * AT(yvel0, jv, kv));
      double cell_vol = AT(volume, j, k);
      double cell_mass = cell_vol * AT(density0, j, k);
      dd_add(&s[0], cell_vol);
      dd_add(&s[1], cell_mass);
      dd_add(&s[2], cell_mass * AT(energy0, j, k));
      dd_add(&s[3], cell_mass * 0.5 * vsqrd);
      dd_add(&s[4], cell_vol * AT(pressure, j, k));
    }
  }
  for (int q = 0; q < 5; ++q) out[q] = s[q].hi + s[q].lo;
}

/* src/serial/PdV.cpp:92-133: kernel, then for the predictor ideal_gas on
 * level 1, a depth-1 pressure halo and revert. */
void oc_pdv(oc_chunk *c, int predict, double dt) {
  oc_pdv_kernel(c, predict, dt);
  if (predict) {
    int fields[15] = {0};
    oc_ideal_gas(c, 1);
    fields[OC_PRESSURE] = 1;
    oc_update_halo(c, fields, 1);
    oc_revert(c);
  }
}

/* driver/advection.cpp:29-105. */
void oc_advection(oc_chunk *c, int advect_x) {
  int fields[15] = {0};
  int direction = advect_x ? 1 : 2;
  fields[OC_ENERGY1] = 1; fields[OC_DENSITY1] = 1; fields[OC_VOL_FLUX_X] = 1; fields[OC_VOL_FLUX_Y] = 1;
  oc_update_halo(c, fields, 2);
  oc_advec_cell(c, 1, direction);
  memset(fields, 0, sizeof fields);
  fields[OC_DENSITY1] = 1; fields[OC_ENERGY1] = 1; fields[OC_XVEL1] = 1; fields[OC_YVEL1] = 1;
  fields[OC_MASS_FLUX_X] = 1; fields[OC_MASS_FLUX_Y] = 1;
  oc_update_halo(c, fields, 2);
  oc_advec_mom(c, 1, 1, direction);
  oc_advec_mom(c, 2, 1, direction);
  direction = advect_x ? 2 : 1;
  oc_advec_cell(c, 2, direction);
  oc_update_halo(c, fields, 2);
  oc_advec_mom(c, 1, 2, direction);
  oc_advec_mom(c, 2, 2, direction);
}

static void record(oc_chunk *c, oc_summary *s, int *n, int max, int step, double time) {
  double out[5];
  oc_field_summary(c, out);
  if (*n < max) {
    s[*n].step = step; s[*n].time = time;
    s[*n].vol = out[0]; s[*n].mass = out[1]; s[*n].ie = out[2]; s[*n].ke = out[3]; s[*n].press = out[4];
  }
  (*n)++;
}

/* driver/start.cpp:43-138, driver/hydro.cpp:46-223, driver/timestep.cpp:37-109. */
int oc_run(oc_chunk *c, const oc_config *cfg, oc_summary *summaries, int max_summaries, int *steps_done,
           double *dt_trace, int dt_trace_len) {
  int n = 0;
  oc_build_field(c);
  oc_initialise_chunk(c, cfg->xmin, cfg->ymin, cfg->xmax, cfg->ymax);
  oc_generate_chunk(c, cfg->number_of_states, cfg->states);
  oc_ideal_gas(c, 0);
  int fields[15] = {0};
  fields[OC_DENSITY0] = 1; fields[OC_ENERGY0] = 1; fields[OC_PRESSURE] = 1; fields[OC_VISCOSITY] = 1;
  fields[OC_DENSITY1] = 1; fields[OC_ENERGY1] = 1; fields[OC_XVEL0] = 1; fields[OC_YVEL0] = 1;
  fields[OC_XVEL1] = 1; fields[OC_YVEL1] = 1;
  oc_update_halo(c, fields, 2);
  double time = 0.0, dt = cfg->dtinit, dtold = cfg->dtinit;
  int step = 0, advect_x = 1;
  record(c, summaries, &n, max_summaries, step, time);
  for (;;) {
    step += 1;
    /* timestep */
    dt = G_BIG;
    oc_ideal_gas(c, 0);
    memset(fields, 0, sizeof fields);
    fields[OC_PRESSURE] = 1; fields[OC_ENERGY0] = 1; fields[OC_DENSITY0] = 1; fields[OC_XVEL0] = 1; fields[OC_YVEL0] = 1;
    oc_update_halo(c, fields, 1);
    oc_viscosity(c);
    memset(fields, 0, sizeof fields);
    fields[OC_VISCOSITY] = 1;
    oc_update_halo(c, fields, 1);
    int control, jldt, kldt, small;
    double dtlp = oc_calc_dt(c, cfg->dtmin, cfg->dtc_safe, cfg->dtu_safe, cfg->dtv_safe, cfg->dtdiv_safe, &control, &jldt, &kldt, &small);
    if (dtlp <= dt) dt = dtlp;
    {
      double a = dtold * cfg->dtrise;
      double m = (a < dt) ? a : dt;
      dt = (cfg->dtmax < m) ? cfg->dtmax : m;
    }
    if (dt < cfg->dtmin) { if (steps_done) *steps_done = step; return -1; }
    dtold = dt;
    if (dt_trace && step - 1 < dt_trace_len) dt_trace[step - 1] = dt;
    oc_pdv(c, 1, dt);
    oc_accelerate(c, dt);
    oc_pdv(c, 0, dt);
    oc_flux_calc(c, dt);
    oc_advection(c, advect_x);
    oc_reset_field(c);
    advect_x = !advect_x;
    time += dt;
    if (cfg->summary_frequency != 0 && step % cfg->summary_frequency == 0) record(c, summaries, &n, max_summaries, step, time);
    if (time + G_SMALL > cfg->end_time || step >= cfg->end_step) {
      record(c, summaries, &n, max_summaries, step, time);
      break;
    }
  }
  if (steps_done) *steps_done = step;
  return n;
}
