// Device restatement of the collision predicate and the collision
// resolutions, written with explicit round-to-nearest FP64 intrinsics in the
// reference's operation order (no FMA contraction), so that a GPU sweep that
// visits pairs in the reference's order reproduces its state bit for bit.
//
//   closest_approach      src/collision.c:63-172
//   collision (impulse)   src/physics.c:545-625
//   merger                src/physics.c:628-708
//   collision_treatment   src/physics.c:1043-1091
//   lose_moonlet          src/structure.c:1077-1087
#pragma once
#include "common.cuh"

namespace ncg {

struct DevState {
      double *x, *y, *z, *vx, *vy, *vz, *m, *R;
      int *ex, *did, *free_idx, *scal;
};

#define DADD __dadd_rn
#define DSUB __dsub_rn
#define DMUL __dmul_rn
#define DDIV __ddiv_rn

struct Approach {
      double t;       // time_until_collision
      double p[6];    // approach[]: heavier body's position first
};

// closest_approach(a, b): 1 when a and b collide within dt.
__device__ __forceinline__ bool d_approach(const DevState &S, int a, int b, double dt, Approach *ap)
{
      if (!(S.ex[a] && S.ex[b])) return false;
      double R_a = S.R[a], R_b = S.R[b];
      double vx_a = S.vx[a], vy_a = S.vy[a], vz_a = S.vz[a];
      double vx_b = S.vx[b], vy_b = S.vy[b], vz_b = S.vz[b];
      double xa = S.x[a], ya = S.y[a], za = S.z[a];
      double xb = S.x[b], yb = S.y[b], zb = S.z[b];
      double dx = DSUB(xa, xb), dy = DSUB(ya, yb), dz = DSUB(za, zb);
      double dvx = DSUB(vx_a, vx_b), dvy = DSUB(vy_a, vy_b), dvz = DSUB(vz_a, vz_b);
      double dr_dot_dv = DADD(DADD(DMUL(dx, dvx), DMUL(dy, dvy)), DMUL(dz, dvz));
      if (dr_dot_dv >= 0.0) return false;
      double dr2 = DADD(DADD(DMUL(dx, dx), DMUL(dy, dy)), DMUL(dz, dz));
      double dv2 = DADD(DADD(DMUL(dvx, dvx), DMUL(dvy, dvy)), DMUL(dvz, dvz));
      double R = DADD(R_a, R_b);
      double disc = DADD(DMUL(dr_dot_dv, dr_dot_dv), DMUL(dv2, DSUB(DMUL(R, R), dr2)));
      if (disc <= 0.0) return false;
      double t = DDIV(-DADD(dr_dot_dv, __dsqrt_rn(disc)), dv2);
      if (t > dt) return false;
      if (ap) {
            ap->t = t;
            xa = DADD(xa, DMUL(t, vx_a)); ya = DADD(ya, DMUL(t, vy_a)); za = DADD(za, DMUL(t, vz_a));
            xb = DADD(xb, DMUL(t, vx_b)); yb = DADD(yb, DMUL(t, vy_b)); zb = DADD(zb, DMUL(t, vz_b));
            if (S.m[a] > S.m[b]) {
                  ap->p[0] = xa; ap->p[1] = ya; ap->p[2] = za; ap->p[3] = xb; ap->p[4] = yb; ap->p[5] = zb;
            } else {
                  ap->p[0] = xb; ap->p[1] = yb; ap->p[2] = zb; ap->p[3] = xa; ap->p[4] = ya; ap->p[5] = za;
            }
      }
      return true;
}

// x^(1/3.) with the double exponent y = 1.0/3.0, correctly rounded.
// y = 1/3 - 1/(3*2^54), so x^y = cbrt(x) * x^delta with delta = -1/(3*2^54):
// cbrt(x) is refined to double-double precision by one Newton step
// (r - (r^3 - x)/(3 r^2), r^3 formed exactly with fma-based products), and
// x^delta = 1 + delta*ln(x) to far below half an ulp; the double-double sum
// is rounded once.
__device__ __forceinline__ double pow_one_third(double x)
{
      if (!(x > 0.) || isinf(x) || x < 2.2250738585072014e-308) return pow(x, 1.0 / 3.0);
      double r = cbrt(x);
      double r2h = r * r;
      double r2l = fma(r, r, -r2h);
      double r3h = r2h * r;
      double r3l = fma(r2h, r, -r3h) + r2l * r;
      double f = (r3h - x) + r3l;           // r^3 - x (r3h - x is exact)
      double c = f / (3.0 * r2h);           // Newton correction
      const double delta = -(1.0 / 3.0) * 0x1p-54;
      double corr = r * (delta * log(x));   // cbrt(x) * (x^delta - 1)
      return r + (corr - c);
}

// lose_moonlet(a)
__device__ __forceinline__ void d_lose(const DevState &S, int a, int mesh_bool)
{
      int nf = S.scal[S_NFREE];
      S.free_idx[nf] = a;
      nf++;
      S.ex[a] = 0;
      if (a <= 2 && mesh_bool) nf--;
      S.scal[S_NFREE] = nf;
}

// collision(a, b, f): impulse exchange, bodies put back at the start of the step
__device__ __forceinline__ void d_impulse(const DevState &S, int a, int b, double f, const Approach &ap,
                                          double *rec)
{
      double R = DADD(S.R[a], S.R[b]);
      double m_a = S.m[a], m_b = S.m[b];
      double vx_a = S.vx[a], vy_a = S.vy[a], vz_a = S.vz[a];
      double vx_b = S.vx[b], vy_b = S.vy[b], vz_b = S.vz[b];
      double xa = ap.p[0], ya = ap.p[1], za = ap.p[2], xb = ap.p[3], yb = ap.p[4], zb = ap.p[5];
      double dr_dot_dv = DADD(DADD(DMUL(DSUB(xa, xb), DSUB(vx_a, vx_b)), DMUL(DSUB(ya, yb), DSUB(vy_a, vy_b))),
                              DMUL(DSUB(za, zb), DSUB(vz_a, vz_b)));
      double alpha = DDIV(DMUL(DMUL(f, m_a), m_b), DMUL(DMUL(DADD(m_a, m_b), R), R));
      double ad = DMUL(alpha, dr_dot_dv);
      double Jx = DMUL(ad, DSUB(xb, xa)), Jy = DMUL(ad, DSUB(yb, ya)), Jz = DMUL(ad, DSUB(zb, za));
      vx_a = DADD(vx_a, DDIV(Jx, m_a)); vy_a = DADD(vy_a, DDIV(Jy, m_a)); vz_a = DADD(vz_a, DDIV(Jz, m_a));
      vx_b = DSUB(vx_b, DDIV(Jx, m_b)); vy_b = DSUB(vy_b, DDIV(Jy, m_b)); vz_b = DSUB(vz_b, DDIV(Jz, m_b));
      double t = ap.t;
      S.x[a] = DSUB(xa, DMUL(t, vx_a)); S.y[a] = DSUB(ya, DMUL(t, vy_a)); S.z[a] = DSUB(za, DMUL(t, vz_a));
      S.vx[a] = vx_a; S.vy[a] = vy_a; S.vz[a] = vz_a;
      S.x[b] = DSUB(xb, DMUL(t, vx_b)); S.y[b] = DSUB(yb, DMUL(t, vy_b)); S.z[b] = DSUB(zb, DMUL(t, vz_b));
      S.vx[b] = vx_b; S.vy[b] = vy_b; S.vz[b] = vz_b;
      if (rec) {
            double dvx = DSUB(vx_a, vx_b), dvy = DSUB(vy_a, vy_b), dvz = DSUB(vz_a, vz_b);
            rec[5] = __dsqrt_rn(DADD(DADD(DMUL(dvx, dvx), DMUL(dvy, dvy)), DMUL(dvz, dvz)));
            rec[6] = dr_dot_dv;
      }
}

// merger(a, b): b merges into a
__device__ __forceinline__ void d_merge(const DevState &S, int a, int b, const Approach &ap, int one_only,
                                        int mesh_bool, double *rec)
{
      const double FOUR_PI = 4. * 3.14159265358979323846;
      double m_a = S.m[a], m_b = S.m[b], R_a = S.R[a], R_b = S.R[b];
      double rho_a = DDIV(DMUL(3., m_a), DMUL(DMUL(DMUL(FOUR_PI, R_a), R_a), R_a));
      double rho_b = DDIV(DMUL(3., m_b), DMUL(DMUL(DMUL(FOUR_PI, R_b), R_b), R_b));
      double m = DADD(m_a, m_b);
      double avg = DDIV(DADD(DMUL(m_a, rho_a), DMUL(m_b, rho_b)), m);
      double vx_a = S.vx[a], vy_a = S.vy[a], vz_a = S.vz[a];
      double vx_b = S.vx[b], vy_b = S.vy[b], vz_b = S.vz[b];
      double v0 = DDIV(DADD(DMUL(m_a, vx_a), DMUL(m_b, vx_b)), m);
      double v1 = DDIV(DADD(DMUL(m_a, vy_a), DMUL(m_b, vy_b)), m);
      double v2 = DDIV(DADD(DMUL(m_a, vz_a), DMUL(m_b, vz_b)), m);
      double r0 = DDIV(DADD(DMUL(m_a, ap.p[0]), DMUL(m_b, ap.p[3])), m);
      double r1 = DDIV(DADD(DMUL(m_a, ap.p[1]), DMUL(m_b, ap.p[4])), m);
      double r2 = DDIV(DADD(DMUL(m_a, ap.p[2]), DMUL(m_b, ap.p[5])), m);
      double t = ap.t;
      S.x[a] = DSUB(r0, DMUL(t, v0)); S.y[a] = DSUB(r1, DMUL(t, v1)); S.z[a] = DSUB(r2, DMUL(t, v2));
      S.vx[a] = v0; S.vy[a] = v1; S.vz[a] = v2;
      S.m[a] = m;
      S.R[a] = pow_one_third(DDIV(DMUL(3.0, m), DMUL(FOUR_PI, avg)));
      d_lose(S, b, mesh_bool);
      S.did[a] = one_only;
      if (rec) {
            double dvx = DSUB(vx_a, vx_b), dvy = DSUB(vy_a, vy_b), dvz = DSUB(vz_a, vz_b);
            rec[5] = __dsqrt_rn(DADD(DADD(DMUL(dvx, dvx), DMUL(dvy, dvy)), DMUL(dvz, dvz)));
            double xa = ap.p[0], ya = ap.p[1], za = ap.p[2], xb = ap.p[3], yb = ap.p[4], zb = ap.p[5];
            rec[6] = DADD(DADD(DMUL(DSUB(xa, xb), dvx), DMUL(DSUB(ya, yb), dvy)), DMUL(DSUB(za, zb), dvz));
      }
}

}  // namespace ncg
