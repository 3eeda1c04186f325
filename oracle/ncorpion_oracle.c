/*
 * TEST INFRASTRUCTURE ONLY - the CPU oracle.  Not part of the product path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it,
 * and only to check or time against the GPU library.
 *
 * A plain-C restatement of NcorpiON's mutual-interaction hot path with the
 * compile-time macros of src/parameters.h turned into a runtime parameter
 * struct (struct ncgpu_params, include/ncgpu.h).  Each function follows the
 * reference function cited beside it, operation for operation (FP64, no FMA
 * contraction: build with -ffp-contract=off), so its results are
 * bit-identical to the reference's own build; tests pin this against the
 * reference compiled from source (oracle/ref_build.py) and against committed
 * golden vectors (tests/golden/).
 *
 * Bodies are `struct moonlet` records: 8 doubles x, y, z, vx, vy, vz, mass,
 * radius (src/structure.h:74-84); exists[] one int per slot.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "../include/ncgpu.h"

typedef struct ncgpu_body body;

/* vector_field, brute-force branch + central mass (src/physics.c:63-266 with
   mesh_bool = 0, J2/tides/perturber off).  acc: 3 doubles per slot. */
void orc_vector_field(int lid, const body *b, const int *ex, const body *cm, const struct ncgpu_params *P,
                      double *acc, double *cm_acc)
{
      int k, p;
      const double G = P->G;
      const double XX = P->central_mass_bool ? cm->x : 0., YY = P->central_mass_bool ? cm->y : 0.,
                   ZZ = P->central_mass_bool ? cm->z : 0.;
      const double M = cm->mass;
      cm_acc[0] = cm_acc[1] = cm_acc[2] = 0.;
      for (k = 0; k <= lid; k++) {
            acc[3 * k] = acc[3 * k + 1] = acc[3 * k + 2] = 0.;
      }
      for (k = 0; k <= lid; k++) {
            if (!ex[k]) continue;
            double X = b[k].x, Y = b[k].y, Z = b[k].z, mk = b[k].mass;
            double DX = X - XX, DY = Y - YY, DZ = Z - ZZ;
            double rk = sqrt(DX * DX + DY * DY + DZ * DZ);
            double r3 = rk * rk * rk;
            double mu = G * M;
            double aX, aY, aZ;
            if (P->central_mass_bool) {            /* src/physics.c:133-146 */
                  aX = -mu * DX / r3;
                  aY = -mu * DY / r3;
                  aZ = -mu * DZ / r3;
                  cm_acc[0] += G * mk * DX / r3;
                  cm_acc[1] += G * mk * DY / r3;
                  cm_acc[2] += G * mk * DZ / r3;
            } else {
                  aX = aY = aZ = 0.;
            }
            if (P->mutual_bool) {                  /* src/physics.c:174-202 */
                  for (p = 0; p < k; p++) {
                        if (!ex[p]) continue;
                        double mp = b[p].mass, Xp = b[p].x, Yp = b[p].y, Zp = b[p].z;
                        double Rp = b[p].radius, Rk = b[k].radius;
                        double dx = X - Xp, dy = Y - Yp, dz = Z - Zp;
                        double soft = P->softening_parameter * (Rk + Rp);
                        double D = sqrt(dx * dx + dy * dy + dz * dz + soft * soft);
                        double D3 = D * D * D;
                        aX -= G * mp * dx / D3;
                        aY -= G * mp * dy / D3;
                        aZ -= G * mp * dz / D3;
                        acc[3 * p] += G * mk * dx / D3;
                        acc[3 * p + 1] += G * mk * dy / D3;
                        acc[3 * p + 2] += G * mk * dz / D3;
                  }
            }
            acc[3 * k] = aX;                        /* src/physics.c:264-266 */
            acc[3 * k + 1] = aY;
            acc[3 * k + 2] = aZ;
      }
}

/* kick (src/rk4.c:68-106): F on a copy, then v += timestep * a. */
void orc_kick(int lid, body *b, const int *ex, body *cm, double dt, const struct ncgpu_params *P)
{
      int i;
      double *acc = (double *)malloc(sizeof(double) * 3 * (size_t)(lid + 1 > 0 ? lid + 1 : 1));
      double cma[3];
      orc_vector_field(lid, b, ex, cm, P, acc, cma);
      for (i = 0; i <= lid; i++) {
            if (!ex[i]) continue;
            b[i].vx += dt * acc[3 * i];
            b[i].vy += dt * acc[3 * i + 1];
            b[i].vz += dt * acc[3 * i + 2];
      }
      if (P->central_mass_bool) {
            cm->vx += dt * cma[0];
            cm->vy += dt * cma[1];
            cm->vz += dt * cma[2];
      }
      free(acc);
}

/* drift (src/rk4.c:109-127): x += timestep * v. */
void orc_drift(int lid, body *b, const int *ex, body *cm, double dt, const struct ncgpu_params *P)
{
      int i;
      for (i = 0; i <= lid; i++) {
            if (!ex[i]) continue;
            b[i].x += dt * b[i].vx;
            b[i].y += dt * b[i].vy;
            b[i].z += dt * b[i].vz;
      }
      if (P->central_mass_bool) {
            cm->x += dt * cm->vx;
            cm->y += dt * cm->vy;
            cm->z += dt * cm->vz;
      }
}
