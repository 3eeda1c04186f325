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
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "../include/ncgpu.h"

typedef struct ncgpu_body body;

/* The J2 contribution of the central body's bulge to body k and to CM_acc
   (src/physics.c:149-160), in the reference's operation order. */
static void j2_terms(const struct ncgpu_params *P, double mu, double M, double DX, double DY, double DZ, double rk,
                     double r3, double mk, double *aX, double *aY, double *aZ, double *cm_acc)
{
      /* J2_value, or the fluid-body J2 of the current central mass
         (src/structure.c:507, src/rk4.c:459-463) */
      double J2 = P->par_J2 != 0. ? P->par_J2
                                  : 0.5 * P->par_sideral_omega * P->par_sideral_omega * P->par_R_unit * P->par_R_unit *
                                            P->par_R_unit / (P->par_G * M);
      double r2 = rk * rk;
      double r5 = r3 * r2;
      double K = mu * P->par_R_unit * P->par_R_unit * J2 / r5;
      *aX += K * (-1.5 * DX + 7.5 / r2 * DZ * DZ * DX);
      *aY += K * (-1.5 * DY + 7.5 / r2 * DZ * DZ * DY);
      *aZ += K * (-4.5 * DZ + 7.5 / r2 * DZ * DZ * DZ);
      cm_acc[0] += K * (1.5 * DX - 7.5 / r2 * DZ * DZ * DX) * mk / M;
      cm_acc[1] += K * (1.5 * DY - 7.5 / r2 * DZ * DZ * DY) * mk / M;
      cm_acc[2] += K * (4.5 * DZ - 7.5 / r2 * DZ * DZ * DZ) * mk / M;
}

/* vector_field, brute-force branch + central mass and J2 (src/physics.c:63-266
   with mesh_bool = 0, tides/perturber off).  acc: 3 doubles per slot. */
void orc_vector_field(int lid, const body *b, const int *ex, const body *cm, const struct ncgpu_params *P,
                      double *acc, double *cm_acc)
{
      int k, p;
      const double G = P->par_G;
      const double XX = P->par_central_mass_bool ? cm->x : 0., YY = P->par_central_mass_bool ? cm->y : 0.,
                   ZZ = P->par_central_mass_bool ? cm->z : 0.;
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
            if (P->par_central_mass_bool) {            /* src/physics.c:133-146 */
                  aX = -mu * DX / r3;
                  aY = -mu * DY / r3;
                  aZ = -mu * DZ / r3;
                  cm_acc[0] += G * mk * DX / r3;
                  cm_acc[1] += G * mk * DY / r3;
                  cm_acc[2] += G * mk * DZ / r3;
            } else {
                  aX = aY = aZ = 0.;
            }
            if (P->par_J2_bool) j2_terms(P, mu, M, DX, DY, DZ, rk, r3, mk, &aX, &aY, &aZ, cm_acc);
            if (P->par_mutual_bool) {                  /* src/physics.c:174-202 */
                  for (p = 0; p < k; p++) {
                        if (!ex[p]) continue;
                        double mp = b[p].mass, Xp = b[p].x, Yp = b[p].y, Zp = b[p].z;
                        double Rp = b[p].radius, Rk = b[k].radius;
                        double dx = X - Xp, dy = Y - Yp, dz = Z - Zp;
                        double soft = P->par_softening_parameter * (Rk + Rp);
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

/* tides (src/physics.c:496-542), constant time lag tides raised on the central
   body, as kick calls them after the vector field (src/rk4.c:88-90).  b is the
   state before the kick, acc (3 per slot) and cm_acc hold the vector field's
   accelerations and receive the tidal terms; the central body's rotation
   P->par_sideral_omega changes body by body in slot order, and the next body's
   terms use the changed value. */
static void port_tides(int lid, const body *b, const int *ex, const body *cm, double dt, struct ncgpu_params *P,
                       double *acc, double *cm_acc)
{
      const double R_unit = P->par_R_unit, Dt = P->par_Delta_t;
      double R5 = R_unit * R_unit * R_unit * R_unit * R_unit;
      double A = 3. * P->par_k2 * P->par_G * R5;
      double M = cm->mass;
      double CMaccX = cm_acc[0], CMaccY = cm_acc[1], CMaccZ = cm_acc[2];
      for (int j = 0; j <= lid; j++) {
            if (!ex[j]) continue;
            double X = b[j].x - cm->x, Y = b[j].y - cm->y, Z = b[j].z - cm->z;
            double vX = b[j].vx - cm->vx + 0.5 * dt * (acc[3 * j] - CMaccX);
            double vY = b[j].vy - cm->vy + 0.5 * dt * (acc[3 * j + 1] - CMaccY);
            double vZ = b[j].vz - cm->vz + 0.5 * dt * (acc[3 * j + 2] - CMaccZ);
            double m = b[j].mass;
            double r2 = X * X + Y * Y + Z * Z;
            double r10 = r2 * r2 * r2 * r2 * r2;
            double rv = X * vX + Y * vY + Z * vZ;
            double r_x_OmX = Y * P->par_sideral_omega;
            double r_x_OmY = -X * P->par_sideral_omega;
            double K = A * m / r10;
            double S = 1. / (1. + m / M);
            double aX = S * K * (r2 * X + Dt * (2. * rv * X + r2 * (vX + r_x_OmX)));
            double aY = S * K * (r2 * Y + Dt * (2. * rv * Y + r2 * (vY + r_x_OmY)));
            double aZ = S * K * (r2 * Z + Dt * (2. * rv * Z + r2 * vZ));
            acc[3 * j] -= aX;
            acc[3 * j + 1] -= aY;
            acc[3 * j + 2] -= aZ;
            cm_acc[0] += aX * m / M;
            cm_acc[1] += aY * m / M;
            cm_acc[2] += aZ * m / M;
            P->par_sideral_omega += dt * m / (P->par_dimensionless_moi * M * R_unit * R_unit) * (X * aY - Y * aX) / S;
      }
}

/* kick (src/rk4.c:68-106): F on a copy, tides, then v += timestep * a.  With
   tides, P->par_sideral_omega is updated. */
void orc_kick(int lid, body *b, const int *ex, body *cm, double dt, struct ncgpu_params *P)
{
      int i;
      double *acc = (double *)malloc(sizeof(double) * 3 * (size_t)(lid + 1 > 0 ? lid + 1 : 1));
      double cma[3];
      orc_vector_field(lid, b, ex, cm, P, acc, cma);
      if (P->par_central_tides_bool) port_tides(lid, b, ex, cm, dt, P, acc, cma);
      for (i = 0; i <= lid; i++) {
            if (!ex[i]) continue;
            b[i].vx += dt * acc[3 * i];
            b[i].vy += dt * acc[3 * i + 1];
            b[i].vz += dt * acc[3 * i + 2];
      }
      if (P->par_central_mass_bool) {
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
      if (P->par_central_mass_bool) {
            cm->x += dt * cm->vx;
            cm->y += dt * cm->vy;
            cm->z += dt * cm->vz;
      }
}

/* ======================================================================== */
/* Collisions and the mesh search.  A single "world" (the reference's global */
/* state, src/structure.c:62-115) lives in this file.                       */
/* ======================================================================== */

static int need_to_reduce_com = 0;  /* need_to_reduce_COM_bool */

static struct {
      struct ncgpu_params P;
      int n_max, lid;
      body *b;
      int *ex, *did, *free_idx;
      int n_free;
      body cm;
      double dt;
      double approach[6], t_coll;
      int *ev;
      int n_ev, ev_cap;
      int collision_count;
      /* mesh */
      double gam;
      int *pairs;
      long n_pairs, pair_cap;
      long total_neighbours;
      int how_many_small, how_many_big;
      /* hash: open addressing map cell index -> head/tail of an insertion-ordered list */
      long *hkey;
      int *hhead, *htail;
      long hcap;
      int *next_in_cell;
      long *used_slots;
      long n_used;
      int three[3];
      int force_naive;  /* force_naive_bool: the mesh run fell back to brute force */
} W;

static void push_event(int a, int b, int type)
{
      if (W.n_ev >= W.ev_cap) {
            W.ev_cap = W.ev_cap ? 2 * W.ev_cap : 1024;
            W.ev = (int *)realloc(W.ev, sizeof(int) * 3 * (size_t)W.ev_cap);
      }
      W.ev[3 * W.n_ev] = a;
      W.ev[3 * W.n_ev + 1] = b;
      W.ev[3 * W.n_ev + 2] = type;
      W.n_ev++;
}

int orc_w_init(int n_max, const struct ncgpu_params *P)
{
      free(W.b); free(W.ex); free(W.did); free(W.free_idx); free(W.pairs); free(W.hkey); free(W.hhead);
      free(W.htail); free(W.next_in_cell); free(W.used_slots); free(W.ev);
      memset(&W, 0, sizeof W);
      W.P = *P;
      W.n_max = n_max;
      W.b = (body *)calloc((size_t)n_max, sizeof(body));
      W.ex = (int *)calloc((size_t)n_max, sizeof(int));
      W.did = (int *)calloc((size_t)n_max, sizeof(int));
      W.free_idx = (int *)calloc((size_t)n_max, sizeof(int));
      W.pair_cap = 5L * n_max * (long)P->par_how_many_neighbours + 64;
      W.pairs = (int *)malloc(sizeof(int) * 2 * (size_t)W.pair_cap);
      W.hcap = 1;
      while (W.hcap < 4L * n_max) W.hcap <<= 1;
      W.hkey = (long *)malloc(sizeof(long) * (size_t)W.hcap);
      W.hhead = (int *)malloc(sizeof(int) * (size_t)W.hcap);
      W.htail = (int *)malloc(sizeof(int) * (size_t)W.hcap);
      for (long s = 0; s < W.hcap; s++) W.hkey[s] = -1;
      W.next_in_cell = (int *)malloc(sizeof(int) * (size_t)n_max);
      W.used_slots = (long *)malloc(sizeof(long) * (size_t)n_max);
      return (W.b && W.ex && W.did && W.pairs && W.hkey) ? 0 : -1;
}

void orc_w_set(int lid, const body *b, const int *ex, const body *cm, double dt, double gam)
{
      int j;
      W.lid = lid;
      memcpy(W.b, b, sizeof(body) * (size_t)(lid + 1));
      for (j = 0; j < W.n_max; j++) {
            W.ex[j] = j <= lid ? ex[j] : 0;
            W.did[j] = 0;
      }
      W.cm = *cm;
      W.dt = dt;
      W.gam = gam;
      W.n_free = 0;
      W.n_ev = 0;
      W.n_pairs = 0;
      W.total_neighbours = 0;
      W.collision_count = 0;
      need_to_reduce_com = 0;
}

void orc_w_set_timestep(double dt) { W.dt = dt; }
void orc_w_set_force_naive(int v) { W.force_naive = v; }
void orc_w_set_gam(double gam) { W.gam = gam; }

int orc_w_get(body *b, int *ex, body *cm)
{
      memcpy(b, W.b, sizeof(body) * (size_t)(W.lid + 1));
      memcpy(ex, W.ex, sizeof(int) * (size_t)(W.lid + 1));
      *cm = W.cm;
      return W.lid;
}

int orc_w_events(int *out, int cap)
{
      int n = W.n_ev < cap ? W.n_ev : cap;
      if (out && n) memcpy(out, W.ev, sizeof(int) * 3 * (size_t)n);
      return W.n_ev;
}
void orc_w_events_reset(void) { W.n_ev = 0; }

long orc_w_pairs(int *out, long cap)
{
      long n = W.n_pairs < cap ? W.n_pairs : cap;
      if (out && n) memcpy(out, W.pairs, sizeof(int) * 2 * (size_t)n);
      return W.n_pairs;
}
long orc_w_total_neighbours(void) { return W.total_neighbours; }
int orc_w_collision_count(void) { return W.collision_count; }

/* lose_moonlet (src/structure.c:1077-1087) */
static void lose(int a)
{
      W.free_idx[W.n_free++] = a;
      W.ex[a] = 0;
      if (a <= 2 && W.P.par_mesh_bool) W.n_free--;
}

/* closest_approach (src/collision.c:63-172); returns 1 and fills W.approach
   and W.t_coll when a and b collide within the timestep. */
static int approach(int a, int b)
{
      if (!(W.ex[a] && W.ex[b])) return 0;
      const body *A = W.b + a, *B = W.b + b;
      double R_a = A->radius, R_b = B->radius;
      double vx_a = A->vx, vy_a = A->vy, vz_a = A->vz, vx_b = B->vx, vy_b = B->vy, vz_b = B->vz;
      double xa = A->x, ya = A->y, za = A->z, xb = B->x, yb = B->y, zb = B->z;
      double dx = xa - xb, dy = ya - yb, dz = za - zb;
      double dvx = vx_a - vx_b, dvy = vy_a - vy_b, dvz = vz_a - vz_b;
      double dr_dot_dv = dx * dvx + dy * dvy + dz * dvz;
      if (dr_dot_dv >= 0.0) return 0;
      double dr2 = dx * dx + dy * dy + dz * dz;
      double dv2 = dvx * dvx + dvy * dvy + dvz * dvz;
      double R = R_a + R_b;
      double disc = dr_dot_dv * dr_dot_dv + dv2 * (R * R - dr2);
      if (disc <= 0.0) return 0;
      double t = -(dr_dot_dv + sqrt(disc)) / dv2;
      W.t_coll = t;
      if (t > W.dt) return 0;
      xa += t * vx_a; ya += t * vy_a; za += t * vz_a;
      xb += t * vx_b; yb += t * vy_b; zb += t * vz_b;
      if (A->mass > B->mass) {
            W.approach[0] = xa; W.approach[1] = ya; W.approach[2] = za;
            W.approach[3] = xb; W.approach[4] = yb; W.approach[5] = zb;
      } else {
            W.approach[0] = xb; W.approach[1] = yb; W.approach[2] = zb;
            W.approach[3] = xa; W.approach[4] = ya; W.approach[5] = za;
      }
      return 1;
}

/* collision (src/physics.c:545-625): impulse with parameter f */
static void impulse(int a, int b, double f)
{
      body *A = W.b + a, *B = W.b + b;
      double R = A->radius + B->radius, m_a = A->mass, m_b = B->mass;
      double vx_a = A->vx, vy_a = A->vy, vz_a = A->vz, vx_b = B->vx, vy_b = B->vy, vz_b = B->vz;
      double xa = W.approach[0], ya = W.approach[1], za = W.approach[2];
      double xb = W.approach[3], yb = W.approach[4], zb = W.approach[5];
      double dr_dot_dv = (xa - xb) * (vx_a - vx_b) + (ya - yb) * (vy_a - vy_b) + (za - zb) * (vz_a - vz_b);
      double alpha = f * m_a * m_b / ((m_a + m_b) * R * R);
      double Jx = alpha * dr_dot_dv * (xb - xa), Jy = alpha * dr_dot_dv * (yb - ya), Jz = alpha * dr_dot_dv * (zb - za);
      vx_a += Jx / m_a; vy_a += Jy / m_a; vz_a += Jz / m_a;
      vx_b -= Jx / m_b; vy_b -= Jy / m_b; vz_b -= Jz / m_b;
      double t = W.t_coll;
      A->x = xa - t * vx_a; A->y = ya - t * vy_a; A->z = za - t * vz_a;
      A->vx = vx_a; A->vy = vy_a; A->vz = vz_a;
      B->x = xb - t * vx_b; B->y = yb - t * vy_b; B->z = zb - t * vz_b;
      B->vx = vx_b; B->vy = vy_b; B->vz = vz_b;
}

/* merger (src/physics.c:628-708) */
static void merge(int a, int b)
{
      body *A = W.b + a, *B = W.b + b;
      double m_a = A->mass, m_b = B->mass, R_a = A->radius, R_b = B->radius;
      double rho_a = 3. * m_a / (4. * M_PI * R_a * R_a * R_a);
      double rho_b = 3. * m_b / (4. * M_PI * R_b * R_b * R_b);
      double m = m_a + m_b;
      double avg = (m_a * rho_a + m_b * rho_b) / m;
      double vt0 = (m_a * A->vx + m_b * B->vx) / m, vt1 = (m_a * A->vy + m_b * B->vy) / m,
             vt2 = (m_a * A->vz + m_b * B->vz) / m;
      double rt0 = (m_a * W.approach[0] + m_b * W.approach[3]) / m;
      double rt1 = (m_a * W.approach[1] + m_b * W.approach[4]) / m;
      double rt2 = (m_a * W.approach[2] + m_b * W.approach[5]) / m;
      double t = W.t_coll;
      A->x = rt0 - t * vt0; A->y = rt1 - t * vt1; A->z = rt2 - t * vt2;
      A->vx = vt0; A->vy = vt1; A->vz = vt2;
      A->mass = m;
      A->radius = pow(3.0 * m / (4.0 * M_PI * avg), 1.0 / 3.0);
      lose(b);
      W.did[a] = W.P.par_one_collision_only_bool;
}

static void fragment(int a, int b);

/* collision_treatment (src/physics.c:1043-1091) */
static void treat(int a, int b, int type)
{
      double m_a = W.b[a].mass, m_b = W.b[b].mass;
      int A = m_a > m_b ? a : b, B = m_a > m_b ? b : a;
      push_event(a, b, type);
      if (!(W.ex[a] && W.ex[b])) return;
      if (type == 0 || type == 1) {
            impulse(A, B, type == 0 ? 2.0 : W.P.par_collision_parameter);
            W.did[a] = W.P.par_one_collision_only_bool;
            W.did[b] = W.P.par_one_collision_only_bool;
            if (W.P.par_mutual_bool && W.P.par_mesh_bool && !W.force_naive) {
                  W.pairs[2 * W.n_pairs] = a;
                  W.pairs[2 * W.n_pairs + 1] = b;
                  W.n_pairs++;
            }
      } else if (type == 2) {
            merge(A, B);
      } else if (type == 3) {
            fragment(A, B);
      }
      W.collision_count++;
}

/* brute_force (src/collision.c:425-456) */
void orc_w_brute_force(void)
{
      int i, j, cur = W.lid;
      for (i = 0; i <= cur; i++) {
            if (!W.ex[i]) continue;
            for (j = i + 1; j <= W.lid; j++) {
                  if (!W.ex[j]) continue;
                  if (approach(i, j) && !W.did[i] && !W.did[j]) treat(i, j, W.P.par_collision_type);
            }
      }
}

/* ---- mesh ------------------------------------------------------------- */

/* the linear cell index of hash_table_cell_index (src/collision.c:175-261):
   -1 outside the cube, else i + j*d + k*d^2 with i = d/2 + 1 + floor(X/gam) */
long orc_cell_index(double X, double Y, double Z, double gam, int d)
{
      double cube = gam * (double)d;
      if (fabs(X) > cube / 2.0 || fabs(Y) > cube / 2.0 || fabs(Z) > cube / 2.0) return -1;
      long i = d / 2 + 1 + (int)floor(X / gam);
      long j = d / 2 + 1 + (int)floor(Y / gam);
      long k = d / 2 + 1 + (int)floor(Z / gam);
      return i + j * (long)d + k * (long)d * d;
}

static long hslot(long key)
{
      unsigned long h = (unsigned long)key * 0x9E3779B97F4A7C15ul;
      long s = (long)(h >> 20) & (W.hcap - 1);
      while (W.hkey[s] != -1 && W.hkey[s] != key) s = (s + 1) & (W.hcap - 1);
      return s;
}

static void hash_clear(void)
{
      for (long u = 0; u < W.n_used; u++) W.hkey[W.used_slots[u]] = -1;
      W.n_used = 0;
}

/* neighbours (src/collision.c:264-316) fused with the pop loop order: the
   ids a query pushes (cells l = 0..26, each newest to oldest) are popped in
   reverse, i.e. cells l = 26..0, each in insertion order.  Fills `out` with
   that pop order and inserts k into its own cell. */
static int query_insert(int k, int *out)
{
      int d = W.P.par_collision_cube_cells;
      long L = orc_cell_index(W.b[k].x, W.b[k].y, W.b[k].z, W.gam, d);
      if (L < 0) return 0;
      int n = 0;
      long dd = (long)d * d;
      for (int l = 26; l >= 0; l--) {
            int di = l % 3 - 1, dj = (l / 3) % 3 - 1, dk = l / 9 - 1;
            long c = L + di + dj * (long)d + dk * dd;
            long s = hslot(c);
            if (W.hkey[s] != c) continue;
            for (int p = W.hhead[s]; p >= 0; p = W.next_in_cell[p])
                  if (W.ex[p]) out[n++] = p;
      }
      long s = hslot(L);
      if (W.hkey[s] != L) {
            W.hkey[s] = L;
            W.hhead[s] = W.htail[s] = k;
            W.used_slots[W.n_used++] = s;
      } else {
            W.next_in_cell[W.htail[s]] = k;
            W.htail[s] = k;
      }
      W.next_in_cell[k] = -1;
      return n;
}

static void add_pair(int a, int b)
{
      if (W.n_pairs < W.pair_cap) {
            W.pairs[2 * W.n_pairs] = a;
            W.pairs[2 * W.n_pairs + 1] = b;
      }
      W.n_pairs++;
}

/* mesh (src/collision.c:324-417) */
void orc_w_mesh(void)
{
      int k, p, cur = W.lid;
      int *nb = (int *)malloc(sizeof(int) * (size_t)(W.lid + 2));
      double gam = W.gam;
      for (k = 0; k <= cur; k++) {
            if (!W.ex[k]) continue;
            double R = W.b[k].radius;
            if (R <= gam) {
                  W.how_many_small++;
                  int n = query_insert(k, nb);
                  for (int q = 0; q < n; q++) {
                        p = nb[q];
                        int hit = approach(p, k);
                        if (!hit || W.did[k] || W.did[p]) {
                              if (W.P.par_mutual_bool) add_pair(k, p);
                        } else {
                              treat(p, k, W.P.par_collision_type);
                        }
                        W.total_neighbours++;
                  }
            } else {
                  W.how_many_big++;
                  for (p = 0; p <= W.lid; p++) {
                        if (!W.ex[p] || p == k) continue;
                        double Rp = W.b[p].radius;
                        if (Rp < gam || (Rp >= gam && p > k)) {
                              int hit = approach(p, k);
                              if (!hit || W.did[k] || W.did[p]) {
                                    if (W.P.par_mutual_bool) add_pair(k, p);
                              } else {
                                    treat(p, k, W.P.par_collision_type);
                              }
                        }
                  }
            }
      }
      free(nb);
}

/* get_neighbours_mesh (src/physics.c:1094-1118) */
void orc_w_get_neighbours_mesh(void)
{
      int k, cur = W.lid;
      int *nb = (int *)malloc(sizeof(int) * (size_t)(W.lid + 2));
      for (k = 0; k <= cur; k++) {
            if (!W.ex[k]) continue;
            int n = query_insert(k, nb);
            for (int q = 0; q < n; q++) {
                  add_pair(k, nb[q]);
                  W.total_neighbours++;
            }
      }
      free(nb);
}

/* end of a mesh pass: hash cleared, counters reset (src/rk4.c:356-364) */
void orc_w_mesh_reset(void)
{
      hash_clear();
      W.n_pairs = 0;
      W.total_neighbours = 0;
      W.how_many_small = W.how_many_big = 0;
}

/* three_largest_moonlets + three_largest_three_first (src/structure.c:914-1063) */
void orc_w_three_largest(int *idx)
{
      int i = 0, j;
      double R_0 = 0., R_1 = 0., R_2 = 0., R = 0.;
      int *t = W.three;
      t[0] = t[1] = t[2] = -1;
      for (j = 0; j <= W.lid; j++) {
            if (!W.ex[j]) continue;
            if (i == 0) {
                  R_0 = W.b[j].radius;
                  t[0] = j;
            } else if (i == 1) {
                  R_1 = W.b[j].radius;
                  if (R_0 > R_1) t[1] = j;
                  else { t[1] = t[0]; t[0] = j; R = R_1; R_1 = R_0; R_0 = R; }
            } else if (i == 2) {
                  R_2 = W.b[j].radius;
                  if (R_1 >= R_2) t[2] = j;
                  else if (R_2 > R_1 && R_2 <= R_0) { t[2] = t[1]; t[1] = j; R = R_2; R_2 = R_1; R_1 = R; }
                  else { t[2] = t[1]; t[1] = t[0]; t[0] = j; R = R_2; R_2 = R_1; R_1 = R_0; R_0 = R; }
            } else {
                  R = W.b[j].radius;
                  if (R > R_0) { t[2] = t[1]; t[1] = t[0]; t[0] = j; R_2 = R_1; R_1 = R_0; R_0 = R; }
                  else if (R > R_1) { t[2] = t[1]; t[1] = j; R_2 = R_1; R_1 = R; }
                  else if (R > R_2) { t[2] = j; R_2 = R; }
            }
            i++;
      }
      idx[0] = t[0]; idx[1] = t[1]; idx[2] = t[2];
      /* three_largest_three_first */
      int first = t[0], second = t[1], third = t[2];
      body buf;
      if (first != 0) {
            if (W.ex[0]) { buf = W.b[0]; W.b[0] = W.b[first]; W.b[first] = buf; }
            else { W.b[0] = W.b[first]; lose(first); W.ex[0] = 1; }
            if (second == 0) second = first;
            else if (third == 0) third = first;
      }
      if (second != 1) {
            if (W.ex[1]) { buf = W.b[1]; W.b[1] = W.b[second]; W.b[second] = buf; }
            else { W.b[1] = W.b[second]; lose(second); W.ex[1] = 1; }
            if (third == 1) third = second;
      }
      if (third != 2) {
            if (W.ex[2]) { buf = W.b[2]; W.b[2] = W.b[third]; W.b[third] = buf; }
            else { W.b[2] = W.b[third]; lose(third); W.ex[2] = 1; }
      }
}

/* ---- end of timestep -------------------------------------------------- */


/* total_momentum (src/structure.c:1193-1227) */
static void total_momentum(double *mom)
{
      const int c = W.P.par_central_mass_bool;
      double X = c ? W.cm.x : 0., Y = c ? W.cm.y : 0., Z = c ? W.cm.z : 0.;
      double vX = c ? W.cm.vx : 0., vY = c ? W.cm.vy : 0., vZ = c ? W.cm.vz : 0.;
      double M = c ? W.cm.mass : 0.;
      mom[0] = M * X; mom[1] = M * Y; mom[2] = M * Z; mom[3] = M * vX; mom[4] = M * vY; mom[5] = M * vZ;
      for (int j = 0; j <= W.lid; j++) {
            if (!W.ex[j]) continue;
            const body *B = W.b + j;
            double m = B->mass;
            M += m;
            mom[0] += m * B->x; mom[1] += m * B->y; mom[2] += m * B->z;
            mom[3] += m * B->vx; mom[4] += m * B->vy; mom[5] += m * B->vz;
      }
      for (int d = 0; d < 6; d++) mom[d] /= M;
}

/* tidy_up (src/structure.c:881-911) */
static void tidy_up(void)
{
      int i = 0, j;
      for (j = 0; j <= W.lid; j++) {
            if (W.ex[j]) {
                  if (j > i) W.b[i] = W.b[j];
                  i++;
            }
      }
      for (j = 0; j <= W.lid; j++) W.ex[j] = j < i ? 1 : 0;
      W.lid = i - 1;
      W.n_free = 0;
}

/* end_of_timestep (src/rk4.c:130-404), the parts on the hot path: dumping to
   the central mass or beyond the outer threshold, COM reduction, did_collide
   reset, tidy_up.  Returns how_many_moonlets. */
int orc_w_end_of_timestep(void)
{
      int j, hm = 0;
      const int c = W.P.par_central_mass_bool;
      double XX = c ? W.cm.x : 0., YY = c ? W.cm.y : 0., ZZ = c ? W.cm.z : 0.;
      for (j = 0; j <= W.lid; j++) {
            if (!W.ex[j]) continue;
            body *B = W.b + j;
            double X = B->x, Y = B->y, Z = B->z, m = B->mass;
            double DX = X - XX, DY = Y - YY, DZ = Z - ZZ;
            int losing = 0;
            if (DX * DX + DY * DY + DZ * DZ < W.P.par_disruption_threshold * W.P.par_disruption_threshold && c) {
                  double vX = B->vx, vY = B->vy, vZ = B->vz;
                  W.cm.mass += m;
                  double M = W.cm.mass;
                  W.cm.x *= (M - m) / M; W.cm.y *= (M - m) / M; W.cm.z *= (M - m) / M;
                  W.cm.vx *= (M - m) / M; W.cm.vy *= (M - m) / M; W.cm.vz *= (M - m) / M;
                  W.cm.x += m * X / M; W.cm.y += m * Y / M; W.cm.z += m * Z / M;
                  W.cm.vx += m * vX / M; W.cm.vy += m * vY / M; W.cm.vz += m * vZ / M;
                  lose(j);
                  losing = 1;
            } else if (DX * DX + DY * DY + DZ * DZ > W.P.par_high_dumping_threshold * W.P.par_high_dumping_threshold) {
                  lose(j);
                  losing = 1;
                  need_to_reduce_com = 1;
            }
            if (!losing) hm++;
      }
      if (need_to_reduce_com && W.P.par_reduce_to_COM_bool) {
            double com[6];
            total_momentum(com);
            if (c) {
                  W.cm.x -= com[0]; W.cm.y -= com[1]; W.cm.z -= com[2];
                  W.cm.vx -= com[3]; W.cm.vy -= com[4]; W.cm.vz -= com[5];
            }
            for (j = 0; j <= W.lid; j++) {
                  if (!W.ex[j]) continue;
                  W.b[j].x -= com[0]; W.b[j].y -= com[1]; W.b[j].z -= com[2];
                  W.b[j].vx -= com[3]; W.b[j].vy -= com[4]; W.b[j].vz -= com[5];
            }
            need_to_reduce_com = 0;
      }
      if (W.P.par_collision_bool && (W.P.par_one_collision_only_bool || W.P.par_collision_type == 3))
            for (j = 0; j <= W.lid; j++) W.did[j] = 0;
      if (hm < 9 * W.lid / 10) tidy_up();
      return hm;
}

/* the world's kick / drift (src/rk4.c:68-127) */
void orc_w_kick(void) { orc_kick(W.lid, W.b, W.ex, &W.cm, W.dt, &W.P); }
/* the world's central-body rotation SideralOmega (changed by tides) */
double orc_w_get_sideral_omega(void) { return W.P.par_sideral_omega; }
void orc_w_set_sideral_omega(double w) { W.P.par_sideral_omega = w; }
void orc_w_drift(void) { orc_drift(W.lid, W.b, W.ex, &W.cm, W.dt, &W.P); }

/* one iteration of integration_brute_force_SABA1's loop (src/rk4.c:906-921):
   kick, collisions, drift, end_of_timestep */
int orc_w_step_brute_force(void)
{
      orc_w_kick();
      if (W.P.par_collision_bool) orc_w_brute_force();
      orc_w_drift();
      return orc_w_end_of_timestep();
}

/* vector_field, mesh branches (src/physics.c:84-109, 205-261, 297-379):
   central mass, the three largest bodies (slots 0-2) against every body,
   their mutual pairs, then pairs[] in list order.  acc: 3 per slot. */
void orc_w_vector_field_mesh(double *acc, double *cm_acc)
{
      int k, p, j;
      const double G = W.P.par_G, sp = W.P.par_softening_parameter;
      const int c = W.P.par_central_mass_bool, mut = W.P.par_mutual_bool;
      const body *b = W.b;
      const int *ex = W.ex;
      double XX = c ? W.cm.x : 0., YY = c ? W.cm.y : 0., ZZ = c ? W.cm.z : 0.;
      double M = W.cm.mass;
      double X0 = 0, Y0 = 0, Z0 = 0, m0 = 0, R0 = 0, X1 = 0, Y1 = 0, Z1 = 0, m1 = 0, R1 = 0, X2 = 0, Y2 = 0, Z2 = 0, m2 = 0, R2 = 0;
      if (ex[0]) { X0 = b[0].x; Y0 = b[0].y; Z0 = b[0].z; m0 = b[0].mass; R0 = b[0].radius; }
      if (ex[1]) { X1 = b[1].x; Y1 = b[1].y; Z1 = b[1].z; m1 = b[1].mass; R1 = b[1].radius; }
      if (ex[2]) { X2 = b[2].x; Y2 = b[2].y; Z2 = b[2].z; m2 = b[2].mass; R2 = b[2].radius; }
      cm_acc[0] = cm_acc[1] = cm_acc[2] = 0.;
      for (k = 0; k <= W.lid; k++) acc[3 * k] = acc[3 * k + 1] = acc[3 * k + 2] = 0.;
      for (k = 0; k <= W.lid; k++) {
            if (!ex[k]) continue;
            double X = b[k].x, Y = b[k].y, Z = b[k].z, mk = b[k].mass;
            double DX = X - XX, DY = Y - YY, DZ = Z - ZZ;
            double rk = sqrt(DX * DX + DY * DY + DZ * DZ), r3 = rk * rk * rk, mu = G * M;
            double aX = 0., aY = 0., aZ = 0.;
            if (c) {
                  aX = -mu * DX / r3; aY = -mu * DY / r3; aZ = -mu * DZ / r3;
                  cm_acc[0] += G * mk * DX / r3; cm_acc[1] += G * mk * DY / r3; cm_acc[2] += G * mk * DZ / r3;
            }
            if (W.P.par_J2_bool) j2_terms(&W.P, mu, M, DX, DY, DZ, rk, r3, mk, &aX, &aY, &aZ, cm_acc);
            if (mut && k > 2) {
                  double Rk = b[k].radius, soft, D, D3;
                  double Xi[3] = {X0, X1, X2}, Yi[3] = {Y0, Y1, Y2}, Zi[3] = {Z0, Z1, Z2}, mi[3] = {m0, m1, m2},
                         Ri[3] = {R0, R1, R2};
                  for (int i = 0; i < 3; i++) {
                        if (!ex[i]) continue;
                        DX = X - Xi[i]; DY = Y - Yi[i]; DZ = Z - Zi[i];
                        soft = sp * (Rk + Ri[i]);
                        D = sqrt(DX * DX + DY * DY + DZ * DZ + soft * soft);
                        D3 = D * D * D;
                        aX -= G * mi[i] * DX / D3; aY -= G * mi[i] * DY / D3; aZ -= G * mi[i] * DZ / D3;
                        acc[3 * i] += G * mk * DX / D3; acc[3 * i + 1] += G * mk * DY / D3; acc[3 * i + 2] += G * mk * DZ / D3;
                  }
            }
            acc[3 * k] = aX; acc[3 * k + 1] = aY; acc[3 * k + 2] = aZ;
      }
      if (!mut) return;
      int pr[3][2] = {{0, 1}, {0, 2}, {1, 2}};
      for (int q = 0; q < 3; q++) {
            int u = pr[q][0], w = pr[q][1];
            if (!(ex[u] && ex[w])) continue;
            double DX = b[u].x - b[w].x, DY = b[u].y - b[w].y, DZ = b[u].z - b[w].z;
            double soft = sp * (b[u].radius + b[w].radius);
            double D = sqrt(DX * DX + DY * DY + DZ * DZ + soft * soft), D3 = D * D * D;
            double mu_ = b[u].mass, mw = b[w].mass;
            acc[3 * u] -= G * mw * DX / D3; acc[3 * u + 1] -= G * mw * DY / D3; acc[3 * u + 2] -= G * mw * DZ / D3;
            acc[3 * w] += G * mu_ * DX / D3; acc[3 * w + 1] += G * mu_ * DY / D3; acc[3 * w + 2] += G * mu_ * DZ / D3;
      }
      for (j = 0; j < W.n_pairs; j++) {
            k = W.pairs[2 * j];
            p = W.pairs[2 * j + 1];
            if (!(ex[k] && ex[p] && k > 2 && p > 2)) continue;
            double DX = b[k].x - b[p].x, DY = b[k].y - b[p].y, DZ = b[k].z - b[p].z;
            double soft = sp * (b[k].radius + b[p].radius);
            double D = sqrt(DX * DX + DY * DY + DZ * DZ + soft * soft), D3 = D * D * D;
            double mk = b[k].mass, mp = b[p].mass;
            acc[3 * k] -= G * mp * DX / D3; acc[3 * k + 1] -= G * mp * DY / D3; acc[3 * k + 2] -= G * mp * DZ / D3;
            acc[3 * p] += G * mk * DX / D3; acc[3 * p + 1] += G * mk * DY / D3; acc[3 * p + 2] += G * mk * DZ / D3;
      }
}

void orc_w_kick_mesh(void)
{
      int i;
      double *acc = (double *)malloc(sizeof(double) * 3 * (size_t)(W.lid + 1 > 0 ? W.lid + 1 : 1));
      double cma[3];
      orc_w_vector_field_mesh(acc, cma);
      if (W.P.par_central_tides_bool) port_tides(W.lid, W.b, W.ex, &W.cm, W.dt, &W.P, acc, cma);
      for (i = 0; i <= W.lid; i++) {
            if (!W.ex[i]) continue;
            W.b[i].vx += W.dt * acc[3 * i];
            W.b[i].vy += W.dt * acc[3 * i + 1];
            W.b[i].vz += W.dt * acc[3 * i + 2];
      }
      if (W.P.par_central_mass_bool) {
            W.cm.vx += W.dt * cma[0];
            W.cm.vy += W.dt * cma[1];
            W.cm.vz += W.dt * cma[2];
      }
      free(acc);
}

/* one iteration of integration_mesh's loop (src/rk4.c:760-790) with a given
   gamma; returns total_neighbours of the pass (for the host's gamma update) */
long orc_w_step_mesh(void)
{
      int idx[3];
      long tn;
      orc_w_mesh_reset();
      if (W.P.par_collision_bool) {
            orc_w_three_largest(idx);
            orc_w_mesh();
      }
      orc_w_drift();
      if (!W.P.par_collision_bool) {
            orc_w_three_largest(idx);
            orc_w_get_neighbours_mesh();
      }
      orc_w_kick_mesh();
      tn = W.total_neighbours;
      orc_w_end_of_timestep();
      orc_w_mesh_reset();
      return tn;
}

/* ---- fragmentation (src/physics.c:710-1040) ----------------------------- */

static int frag_error = 0;  /* nonzero where the reference would abort */

static struct {
      int N_tilde, pq[4];
      double mu, nu, C1, k, merging_threshold, fragment_threshold;
      int merger_count, super_catastrophic_count, half_count, full_count;
} F = {15, {-1, 3, -1, 1}, 0.55, 0.4, 1.5, 0.2, 0.0002, 1.5e-8, 0, 0, 0, 0};

void orc_w_set_fragmentation(int N_tilde, const int *pq, double mu, double nu, double C1, double k,
                             double merging_threshold, double fragment_threshold)
{
      F.N_tilde = N_tilde;
      memcpy(F.pq, pq, sizeof F.pq);
      F.mu = mu; F.nu = nu; F.C1 = C1; F.k = k;
      F.merging_threshold = merging_threshold;
      F.fragment_threshold = fragment_threshold;
      F.merger_count = F.super_catastrophic_count = F.half_count = F.full_count = 0;
      frag_error = 0;
}

void orc_w_fragment_counts(int *out)
{
      out[0] = F.merger_count; out[1] = F.super_catastrophic_count; out[2] = F.half_count; out[3] = F.full_count;
}

/* get_free_index (src/structure.c:849-878): 0 on success, -1 past N_max */
static int free_index(int at_end, int *index)
{
      int idx;
      if (W.n_free == 0 || at_end) {
            W.lid += 1;
            idx = W.lid;
            if (idx == W.n_max) return -1;
      } else {
            W.n_free -= 1;
            idx = W.free_idx[W.n_free];
            if (idx > W.lid) W.lid = idx;
      }
      if (W.ex[idx]) return -2;
      W.ex[idx] = 1;
      *index = idx;
      return 0;
}

int orc_w_fragment_error(void) { return frag_error; }

static void fragment(int a, int b)
{
      const double stigma = (3. * F.mu - 1.) / (3. * F.mu);
      body *A = W.b + a, *B = W.b + b;
      double R_2 = A->radius, R_1 = B->radius, R = R_1 + R_2;
      double m_2 = A->mass, m_1 = B->mass, M = m_1 + m_2;
      double rho_1 = 3. * m_1 / (4. * M_PI * R_1 * R_1 * R_1);
      double rho_2 = 3. * m_2 / (4. * M_PI * R_2 * R_2 * R_2);
      double average_density = (m_1 * rho_1 + m_2 * rho_2) / M;
      double rho_12 = rho_1 / rho_2;
      double rho_12_3nu = pow(rho_12, 3. * F.nu);
      double vx_a = A->vx, vy_a = A->vy, vz_a = A->vz, vx_b = B->vx, vy_b = B->vy, vz_b = B->vz;
      double xa = W.approach[0], ya = W.approach[1], za = W.approach[2];
      double xb = W.approach[3], yb = W.approach[4], zb = W.approach[5];
      double dx = xa - xb, dy = ya - yb, dz = za - zb;
      double dvx = vx_a - vx_b, dvy = vy_a - vy_b, dvz = vz_a - vz_b;
      double dr_dot_dv = dx * dvx + dy * dvy + dz * dvz;
      double dv_norm = sqrt(dvx * dvx + dvy * dvy + dvz * dvz);
      double costheta = -dr_dot_dv / (R * dv_norm);
      double costheta3mu = pow(costheta, 3. * F.mu);
      double R_eq = pow(3. * M / (4. * M_PI * average_density), 1. / 3.);
      double vesc = sqrt(2. * W.P.par_G * M / R_eq);
      double K = 3. * F.k * m_1 / (4. * M_PI) / rho_12 * costheta3mu;
      double m_check = K * (pow(F.C1 * dv_norm / vesc, 3. * F.mu) * rho_12_3nu - 1.);
      double m_tilde = M - m_check;
      double m_tilde_2 = m_check / (double)F.N_tilde;
      double v_cm[3], r_cm[3], r_tilde[3], v_tilde[3];
      double t = W.t_coll;
      v_cm[0] = (m_2 * vx_a + m_1 * vx_b) / M; v_cm[1] = (m_2 * vy_a + m_1 * vy_b) / M; v_cm[2] = (m_2 * vz_a + m_1 * vz_b) / M;
      r_cm[0] = (m_2 * xa + m_1 * xb) / M; r_cm[1] = (m_2 * ya + m_1 * yb) / M; r_cm[2] = (m_2 * za + m_1 * zb) / M;

      if (m_check <= F.merging_threshold * M) {  /* merger */
            merge(a, b);
            F.merger_count++;
            return;
      }
      if (m_tilde < 0.1 * M) {  /* super-catastrophic */
            m_tilde = 0.1 * M * pow(1.0 / 0.9 * m_check / M, -1.5);
            A->vx = v_cm[0]; A->vy = v_cm[1]; A->vz = v_cm[2];
            A->x = r_cm[0] - t * v_cm[0]; A->y = r_cm[1] - t * v_cm[1]; A->z = r_cm[2] - t * v_cm[2];
            A->mass = m_tilde;
            A->radius = pow(3. * m_tilde / (4. * M_PI * average_density), 1. / 3.);
            need_to_reduce_com = 1;
            lose(b);
            W.did[a] = W.P.par_one_collision_only_bool;
            F.super_catastrophic_count++;
            double discarded_mass = M - m_tilde;
            if (m_tilde < F.fragment_threshold / 4.) {
                  lose(a);
                  discarded_mass = M;
            }
            if (W.P.par_central_mass_bool) W.cm.mass += discarded_mass;
            return;
      }
      if (m_tilde_2 < F.fragment_threshold && m_check <= m_tilde) {  /* partial fragmentation */
            double r_k[3], v_k[3];
            double v_k_scalar = vesc / stigma * (m_check + K) / m_check * (1.0 - pow(K / (K + m_check), stigma));
            if (v_k_scalar < vesc) { frag_error = 1; return; }
            double in_front_of = v_k_scalar / R;
            r_k[0] = -dx; r_k[1] = -dy; r_k[2] = -dz;
            v_k[0] = in_front_of * r_k[0]; v_k[1] = in_front_of * r_k[1]; v_k[2] = in_front_of * r_k[2];
            double R_tilde = pow(3.0 * m_tilde / (4.0 * M_PI * average_density), 1.0 / 3.0);
            double R_check = pow(3.0 * m_check / (4.0 * M_PI * average_density), 1.0 / 3.0);
            double R_tilde12 = R_tilde + R_check;
            double dr_norm = sqrt(r_k[0] * r_k[0] + r_k[1] * r_k[1] + r_k[2] * r_k[2]);
            r_k[0] *= R_tilde12 / dr_norm; r_k[1] *= R_tilde12 / dr_norm; r_k[2] *= R_tilde12 / dr_norm;
            for (int d = 0; d < 3; d++) {
                  r_tilde[d] = r_cm[d] - m_check / M * r_k[d];
                  v_tilde[d] = v_cm[d] - m_check / M * v_k[d];
            }
            A->x = r_tilde[0] - t * v_tilde[0]; A->y = r_tilde[1] - t * v_tilde[1]; A->z = r_tilde[2] - t * v_tilde[2];
            A->vx = v_tilde[0]; A->vy = v_tilde[1]; A->vz = v_tilde[2];
            A->mass = m_tilde; A->radius = R_tilde;
            B->x = r_tilde[0] + r_k[0] - t * (v_tilde[0] + v_k[0]);
            B->y = r_tilde[1] + r_k[1] - t * (v_tilde[1] + v_k[1]);
            B->z = r_tilde[2] + r_k[2] - t * (v_tilde[2] + v_k[2]);
            B->vx = v_tilde[0] + v_k[0]; B->vy = v_tilde[1] + v_k[1]; B->vz = v_tilde[2] + v_k[2];
            B->mass = m_check; B->radius = R_check;
            if (W.P.par_mutual_bool && W.P.par_mesh_bool && !W.force_naive) add_pair(a, b);
            W.did[a] = W.P.par_one_collision_only_bool;
            W.did[b] = W.P.par_one_collision_only_bool;
            F.half_count++;
            return;
      }
      /* full fragmentation: the tail is N_tilde bodies on a (p, q) lattice */
      int NT = F.N_tilde, n = 0;
      double *r_k = (double *)malloc(sizeof(double) * 3 * (size_t)NT);
      double *v_k = (double *)malloc(sizeof(double) * 3 * (size_t)NT);
      int *id = (int *)malloc(sizeof(int) * (size_t)(NT + 1));
      double dr[3], dv[3], u[3], v[3];
      double R_tilde = pow(3.0 * m_tilde / (4.0 * M_PI * average_density), 1.0 / 3.0);
      double R_tilde_2 = pow(3.0 * m_tilde_2 / (4.0 * M_PI * average_density), 1.0 / 3.0);
      double R_tilde12 = R_tilde + R_tilde_2;
      dr[0] = -dx; dr[1] = -dy; dr[2] = -dz;
      dv[0] = -dvx; dv[1] = -dvy; dv[2] = -dvz;
      double dr_norm = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
      dr[0] *= R_tilde12 / dr_norm; dr[1] *= R_tilde12 / dr_norm; dr[2] *= R_tilde12 / dr_norm;
      double dxv[3] = {dr[1] * dv[2] - dr[2] * dv[1], dr[2] * dv[0] - dr[0] * dv[2], dr[0] * dv[1] - dr[1] * dv[0]};
      double dxv_norm = sqrt(dxv[0] * dxv[0] + dxv[1] * dxv[1] + dxv[2] * dxv[2]);
      if (dxv_norm > 1.0e-5) {
            v[0] = dxv[0] / dxv_norm; v[1] = dxv[1] / dxv_norm; v[2] = dxv[2] / dxv_norm;
      } else {
            /* maximum(|dr0|, |dr1|, |dr2|), src/structure.c:1090-1111 */
            double f0 = fabs(dr[0]), f1 = fabs(dr[1]), f2 = fabs(dr[2]), mx;
            int mm;
            if (f0 >= f1) { mm = 0; mx = f0; } else { mm = 1; mx = f1; }
            if (!(mx >= f2)) mm = 2;
            double num;
            if (mm == 0) {
                  num = dr[1] + dr[2];
                  v[1] = 1.0 / sqrt(2.0 + num * num / (dr[0] * dr[0])); v[2] = v[1]; v[0] = -v[1] * num / dr[0];
            } else if (mm == 1) {
                  num = dr[0] + dr[2];
                  v[0] = 1.0 / sqrt(2.0 + num * num / (dr[1] * dr[1])); v[2] = v[0]; v[1] = -v[0] * num / dr[1];
            } else {
                  num = dr[0] + dr[1];
                  v[0] = 1.0 / sqrt(2.0 + num * num / (dr[2] * dr[2])); v[1] = v[0]; v[2] = -v[0] * num / dr[2];
            }
      }
      double vxd[3] = {v[1] * dr[2] - v[2] * dr[1], v[2] * dr[0] - v[0] * dr[2], v[0] * dr[1] - v[1] * dr[0]};
      u[0] = vxd[0] / R_tilde12; u[1] = vxd[1] / R_tilde12; u[2] = vxd[2] / R_tilde12;
      for (int p = F.pq[0]; p <= F.pq[1]; p++) {
            for (int q = F.pq[2]; q <= F.pq[3]; q++) {
                  double tp = ((double)(2 * p)) * R_tilde_2, tq = ((double)(2 * q)) * R_tilde_2;
                  r_k[3 * n] = dr[0] + tp * u[0] + tq * v[0];
                  r_k[3 * n + 1] = dr[1] + tp * u[1] + tq * v[1];
                  r_k[3 * n + 2] = dr[2] + tp * u[2] + tq * v[2];
                  double zk = pow(1.0 - ((double)n) * m_tilde_2 / (K + m_check), stigma);
                  double zk1 = pow(1.0 - ((double)n + 1.) * m_tilde_2 / (K + m_check), stigma);
                  double vks = vesc / stigma * (m_check + K) / m_tilde_2 * (zk - zk1);
                  if (vks < vesc) frag_error = 2;
                  double iff = vks / sqrt(1.0 + ((double)p) * ((double)p) + ((double)q) * ((double)q));
                  v_k[3 * n] = iff * (dr[0] / R_tilde12 + ((double)p) * u[0] + ((double)q) * v[0]);
                  v_k[3 * n + 1] = iff * (dr[1] / R_tilde12 + ((double)p) * u[1] + ((double)q) * v[1]);
                  v_k[3 * n + 2] = iff * (dr[2] / R_tilde12 + ((double)p) * u[2] + ((double)q) * v[2]);
                  n++;
            }
      }
      double corr[6] = {0., 0., 0., 0., 0., 0.};
      for (n = 0; n < NT; n++) {
            corr[0] += r_k[3 * n]; corr[1] += r_k[3 * n + 1]; corr[2] += r_k[3 * n + 2];
            corr[3] += v_k[3 * n]; corr[4] += v_k[3 * n + 1]; corr[5] += v_k[3 * n + 2];
      }
      for (int d = 0; d < 3; d++) {
            r_tilde[d] = r_cm[d] - m_tilde_2 / M * corr[d];
            v_tilde[d] = v_cm[d] - m_tilde_2 / M * corr[3 + d];
      }
      id[0] = a;
      for (n = 1; n <= NT; n++)
            if (free_index(W.P.par_mesh_bool && !W.force_naive, &id[n]) != 0) frag_error = 3;
      if (W.P.par_mutual_bool && W.P.par_mesh_bool && !W.force_naive)
            for (int p = 0; p <= NT; p++)
                  for (int q = 0; q < p; q++) add_pair(id[p], id[q]);
      lose(b);
      for (n = 0; n <= NT; n++) W.did[id[n]] = W.P.par_one_collision_only_bool;
      body *L0 = W.b + id[0];
      L0->x = r_tilde[0] - t * v_tilde[0]; L0->y = r_tilde[1] - t * v_tilde[1]; L0->z = r_tilde[2] - t * v_tilde[2];
      L0->vx = v_tilde[0]; L0->vy = v_tilde[1]; L0->vz = v_tilde[2];
      L0->mass = m_tilde; L0->radius = R_tilde;
      for (n = 0; n < NT; n++) {
            body *Fk = W.b + id[n + 1];
            Fk->x = r_tilde[0] + r_k[3 * n] - t * (v_tilde[0] + v_k[3 * n]);
            Fk->y = r_tilde[1] + r_k[3 * n + 1] - t * (v_tilde[1] + v_k[3 * n + 1]);
            Fk->z = r_tilde[2] + r_k[3 * n + 2] - t * (v_tilde[2] + v_k[3 * n + 2]);
            Fk->vx = v_tilde[0] + v_k[3 * n]; Fk->vy = v_tilde[1] + v_k[3 * n + 1]; Fk->vz = v_tilde[2] + v_k[3 * n + 2];
            Fk->mass = m_tilde_2; Fk->radius = R_tilde_2;
      }
      F.full_count++;
      free(r_k); free(v_k); free(id);
}

/* ---- output text (src/display.c:321-349) --------------------------------- */

/* display()'s per-value output, fprintf(file, "%.14lf ", v), for the n values
   of v into the file at `path`, then one newline: the CPU baseline of the
   device formatter.  Returns the bytes written, or -1. */
long orc_fprintf_values(const double *v, long n, const char *path)
{
      FILE *f = fopen(path, "w");
      if (!f) return -1;
      for (long i = 0; i < n; i++) fprintf(f, "%.14lf ", v[i]);
      fprintf(f, "\n");
      long bytes = ftell(f);
      fclose(f);
      return bytes;
}

/* ---- elliptic elements (cart2ell, src/structure.c:172-284) ---------------- */

/* cart2ell of body b with the central body cm (CM_buffer) and the
   parameter mu, into alkhqp (a, lambda, k, h, q, p), operation for operation;
   J2 is the J2 in force (the reference's global).  Prints the reference's
   (k, h) warning to stdout when it would (src/structure.c:253-255) and
   returns 1 then, else 0. */
int orc_cart2ell(const body *b, const body *cm, double mu, const struct ncgpu_params *P, double J2, double *alkhqp)
{
      const int central = P->par_central_mass_bool != 0;
      double X = b->x - (central ? cm->x : 0.), Y = b->y - (central ? cm->y : 0.), Z = b->z - (central ? cm->z : 0.);
      double vX = b->vx - (central ? cm->vx : 0.), vY = b->vy - (central ? cm->vy : 0.);
      double vZ = b->vz - (central ? cm->vz : 0.);
      int warned = 0;
      /* semi-major axis, Kepler's third law corrected for J2 on elliptic orbits */
      const double R = sqrt(X * X + Y * Y + Z * Z);
      double V2 = vX * vX + vY * vY + vZ * vZ;
      double AA = R * mu / (2. * mu - R * V2);
      if (P->par_J2_bool && AA > 0. && central) {
            mu *= 1. + 1. * J2 * P->par_R_unit * P->par_R_unit / (AA * AA);
            AA = R * mu / (2. * mu - R * V2);
      }
      alkhqp[0] = AA;
      /* velocities in units of sqrt(mu); angular momentum C */
      const double SMU = sqrt(mu);
      vX /= SMU;
      vY /= SMU;
      vZ /= SMU;
      V2 = vX * vX + vY * vY + vZ * vZ;
      const double RV = X * vX + Y * vY + Z * vZ;
      const double C1 = Y * vZ - Z * vY, C2 = Z * vX - X * vZ, C3 = X * vY - Y * vX;
      const double CC = C1 * C1 + C2 * C2 + C3 * C3;
      const double DC = sqrt(CC);
      const double aux0 = sqrt(2. * (CC + DC * C3));
      alkhqp[4] = aux0 == 0. ? 0. : -C2 / aux0;
      alkhqp[5] = aux0 == 0. ? 0. : C1 / aux0;
      if (R == 0. || V2 == 0.) {
            alkhqp[1] = alkhqp[2] = alkhqp[3] = 0.;
            return 0;
      }
      const double a11 = V2 - 1. / R, a12 = RV / (R * DC), a21 = -RV, a22 = DC - R / DC;
      const double c11 = X * a11 + vX * a21, c12 = X * a12 + vX * a22;
      const double c21 = Y * a11 + vY * a21, c22 = Y * a12 + vY * a22;
      const double FAC1 = C1 / (DC + C3), FAC2 = C2 / (DC + C3);
      const double K1 = c11 - FAC1 * (Z * a11 + vZ * a21);
      const double H1 = -c12 + FAC1 * (Z * a12 + vZ * a22);
      const double H2 = c21 - FAC2 * (Z * a11 + vZ * a21);
      const double K2 = c22 - FAC2 * (Z * a12 + vZ * a22);
      if (fabs(H1 - H2) + fabs(K1 - K2) > 1.e-6) {
            printf("Warning : Bad computation of (k,h) in function cart2ell. (K1 - K2, H1 - H2) = (%.13lf, %.13lf)\n",
                   K1 - K2, H1 - H2);
            warned = 1;
      }
      const double K = 0.5 * (K1 + K2), H = 0.5 * (H1 + H2);
      alkhqp[2] = K;
      alkhqp[3] = H;
      /* mean longitude: elliptic branch, else (NaN square root) hyperbolic */
      double USQA = sqrt(2. / R - V2);
      if (USQA >= 0.) {
            const double b12 = vX - FAC1 * vZ, b22 = vY - FAC2 * vZ;
            const double aux1 = (R * V2 - 1.) / (1. + DC * USQA);
            const double sinF = -b12 * R * USQA + H * aux1, cosF = b22 * R * USQA + K * aux1;
            alkhqp[1] = atan2(sinF, cosF) - RV * USQA;
      } else {
            USQA = sqrt(-(2. / R - V2));
            const double E = atanh(RV * USQA / (R * V2 - 1.));
            alkhqp[1] = sqrt(K * K + H * H) * sinh(E) - E + atan2(H, K);
      }
      return warned;
}

/* display()'s elliptic values (src/display.c:321-347): cart2ell of every
   existing slot <= lid with mu + G m, into out (six blocks a, lambda, k, h,
   q, p of n_existing values).  Returns n_existing. */
long orc_cart2ell_all(int lid, const body *b, const int *ex, const body *cm, double mu,
                      const struct ncgpu_params *P, double J2, double *out, long cap)
{
      long n = 0;
      for (int p = 0; p <= lid; p++) n += ex[p] ? 1 : 0;
      if (6 * n > cap) return -1;
      long j = 0;
      for (int p = 0; p <= lid; p++) {
            if (!ex[p]) continue;
            double alk[6];
            orc_cart2ell(b + p, cm, mu + P->par_G * b[p].mass, P, J2, alk);
            for (int f = 0; f < 6; f++) out[f * n + j] = alk[f];
            j++;
      }
      fflush(stdout);
      return n;
}
