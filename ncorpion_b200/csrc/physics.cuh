// Device restatement of the collision predicate and the collision
// resolutions, written with explicit round-to-nearest FP64 intrinsics in the
// reference's operation order (no FMA contraction), so that a GPU sweep that
// visits pairs in the reference's order reproduces its state bit for bit.
//
//   closest_approach      src/collision.c:63-172
//   collision (impulse)   src/physics.c:545-625
//   merger                src/physics.c:628-708
//   collision_treatment   src/physics.c:1043-1091
//   fragmentation         src/physics.c:710-1040
//   lose_moonlet          src/structure.c:1077-1087
//   get_free_index        src/structure.c:849-878
//   cross_product         src/structure.c:1066-1074
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

// The collision test of closest_approach on the two bodies' values: true
// when they collide within dt, with *t the time of contact (src/collision.c:101-160).
__device__ __forceinline__ bool d_contact(double xa, double ya, double za, double vx_a, double vy_a, double vz_a,
                                          double R_a, double xb, double yb, double zb, double vx_b, double vy_b,
                                          double vz_b, double R_b, double dt, double *t_out)
{
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
      *t_out = t;
      return true;
}

// closest_approach(a, b): 1 when a and b collide within dt.
__device__ __forceinline__ bool d_approach(const DevState &S, int a, int b, double dt, Approach *ap)
{
      if (!(S.ex[a] && S.ex[b])) return false;
      double vx_a = S.vx[a], vy_a = S.vy[a], vz_a = S.vz[a];
      double vx_b = S.vx[b], vy_b = S.vy[b], vz_b = S.vz[b];
      double xa = S.x[a], ya = S.y[a], za = S.z[a];
      double xb = S.x[b], yb = S.y[b], zb = S.z[b];
      double t;
      if (!d_contact(xa, ya, za, vx_a, vy_a, vz_a, S.R[a], xb, yb, zb, vx_b, vy_b, vz_b, S.R[b], dt, &t)) return false;
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

// One body's fields in a cell-ordered copy (64 bytes): the mesh pass reads
// partners from it instead of gathering each field from the state arrays.
struct __align__(16) MRec {
      double x, y, z, R, vx, vy, vz;
      int ex, did;
};

// A record in four 16-byte loads.
__device__ __forceinline__ MRec load_mrec(const MRec *__restrict__ rec, long q)
{
      const double2 *p = reinterpret_cast<const double2 *>(rec + q);
      const double2 a = p[0], b = p[1], c = p[2];
      const int4 d = reinterpret_cast<const int4 *>(rec + q)[3];
      MRec r;
      r.x = a.x; r.y = a.y; r.z = b.x; r.R = b.y; r.vx = c.x; r.vy = c.y;
      r.vz = __longlong_as_double(((long long)(unsigned)d.y << 32) | (unsigned)d.x);
      r.ex = d.z;
      r.did = d.w;
      return r;
}

__device__ __forceinline__ bool d_contact_rec(const MRec &a, const MRec &b, double dt)
{
      double t;
      return a.ex && b.ex && d_contact(a.x, a.y, a.z, a.vx, a.vy, a.vz, a.R, b.x, b.y, b.z, b.vx, b.vy, b.vz, b.R, dt, &t);
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

// get_free_index(at_end): a freed slot (the top of the free stack) or a new
// slot past largest_id; -1 (with ERR_NMAX) when that would reach N_max.
__device__ __forceinline__ int d_free_index(const DevState &S, int at_end, int n_max, unsigned *err)
{
      int idx;
      int nf = S.scal[S_NFREE];
      if (nf == 0 || at_end) {
            idx = S.scal[S_LID] + 1;
            if (idx >= n_max) {
                  atomicOr(err, ERR_NMAX);
                  return -1;
            }
            S.scal[S_LID] = idx;
      } else {
            nf -= 1;
            S.scal[S_NFREE] = nf;
            idx = S.free_idx[nf];
            if (idx > S.scal[S_LID]) S.scal[S_LID] = idx;
      }
      if (S.ex[idx]) {  // the reference aborts: "This index is not free"
            atomicOr(err, ERR_INTERNAL);
            return -1;
      }
      S.ex[idx] = 1;
      return idx;
}

// Constants of the fragmentation model and the driver switches it reads.
struct FragArgs {
      int N_tilde;
      int pq[4];
      double mu, nu, C1, k, merging_threshold, fragment_threshold, G;
      int central_mass_bool;
      int at_end;       // mesh_bool && !force_naive_bool: fragments go past largest_id
      int mesh_bool;    // lose_moonlet's rule for slots 0-2
      int one_only;     // one_collision_only_bool
      int n_max;
      double *cm;       // device central body (x, y, z, vx, vy, vz, mass, radius)
};

// Outcome of one fragmentation: 0 merger, 1 super-catastrophic, 2 partial
// (ids = a, b: the pair (a, b) enters pairs[] in mesh mode), 3 full (ids =
// id[0..N_tilde]: a, then the tail fragments in creation order).
struct FragOut {
      int outcome;
      int nids;
      int ids[NCGPU_MAX_N_TILDE + 1];
};

__device__ __forceinline__ void d_cross(double u1, double u2, double u3, double v1, double v2, double v3, double *w)
{
      w[0] = DSUB(DMUL(u2, v3), DMUL(u3, v2));
      w[1] = DSUB(DMUL(u3, v1), DMUL(u1, v3));
      w[2] = DSUB(DMUL(u1, v2), DMUL(u2, v1));
}

// One tail fragment's offsets (r_k, v_k) relative to the largest fragment, at
// lattice point (p, q) with running index n (the body of the reference's
// (p, q) loop).  Returns false when its speed is below the escape velocity.
__device__ __forceinline__ bool d_tail(int n, int p, int q, const double *dr, const double *u, const double *v,
                                       double R_tilde_2, double R_tilde12, double m_tilde_2, double K,
                                       double m_check, double stigma, double vesc, double *rk, double *vk)
{
      const double tp = DMUL((double)(2 * p), R_tilde_2), tq = DMUL((double)(2 * q), R_tilde_2);
      for (int d = 0; d < 3; d++) rk[d] = DADD(DADD(dr[d], DMUL(tp, u[d])), DMUL(tq, v[d]));
      const double Km = DADD(K, m_check);
      const double zk = pow(DSUB(1.0, DDIV(DMUL((double)n, m_tilde_2), Km)), stigma);
      const double zk1 = pow(DSUB(1.0, DDIV(DMUL(DADD((double)n, 1.), m_tilde_2), Km)), stigma);
      const double vks = DMUL(DDIV(DMUL(DDIV(vesc, stigma), DADD(m_check, K)), m_tilde_2), DSUB(zk, zk1));
      const double pp = (double)p, qq = (double)q;
      const double iff = DDIV(vks, __dsqrt_rn(DADD(DADD(1.0, DMUL(pp, pp)), DMUL(qq, qq))));
      for (int d = 0; d < 3; d++)
            vk[d] = DMUL(iff, DADD(DADD(DDIV(dr[d], R_tilde12), DMUL(pp, u[d])), DMUL(qq, v[d])));
      return !(vks < vesc);
}

// fragmentation(a, b): a is the heavier body (the target), b the impactor.
// General powers use CUDA's pow (the reference uses libm's); the cube roots
// use pow_one_third.  rec (if given) receives DeltaV, dr.dv and m_tilde.
__device__ inline void d_fragment(const DevState &S, int a, int b, const Approach &ap, const FragArgs &F, double *rec,
                           FragOut &out, unsigned *err)
{
      const double FOUR_PI = 4. * 3.14159265358979323846;
      const double stigma = DDIV(DSUB(DMUL(3., F.mu), 1.), DMUL(3., F.mu));
      const double R_2 = S.R[a], R_1 = S.R[b], R = DADD(R_1, R_2);
      const double m_2 = S.m[a], m_1 = S.m[b], M = DADD(m_1, m_2);
      const double rho_1 = DDIV(DMUL(3., m_1), DMUL(DMUL(DMUL(FOUR_PI, R_1), R_1), R_1));
      const double rho_2 = DDIV(DMUL(3., m_2), DMUL(DMUL(DMUL(FOUR_PI, R_2), R_2), R_2));
      const double avg = DDIV(DADD(DMUL(m_1, rho_1), DMUL(m_2, rho_2)), M);
      const double rho_12 = DDIV(rho_1, rho_2);
      const double rho_12_3nu = pow(rho_12, DMUL(3., F.nu));
      const double vx_a = S.vx[a], vy_a = S.vy[a], vz_a = S.vz[a];
      const double vx_b = S.vx[b], vy_b = S.vy[b], vz_b = S.vz[b];
      const double xa = ap.p[0], ya = ap.p[1], za = ap.p[2], xb = ap.p[3], yb = ap.p[4], zb = ap.p[5];
      const double dx = DSUB(xa, xb), dy = DSUB(ya, yb), dz = DSUB(za, zb);
      const double dvx = DSUB(vx_a, vx_b), dvy = DSUB(vy_a, vy_b), dvz = DSUB(vz_a, vz_b);
      const double dr_dot_dv = DADD(DADD(DMUL(dx, dvx), DMUL(dy, dvy)), DMUL(dz, dvz));
      const double dv_norm = __dsqrt_rn(DADD(DADD(DMUL(dvx, dvx), DMUL(dvy, dvy)), DMUL(dvz, dvz)));
      const double costheta = DDIV(-dr_dot_dv, DMUL(R, dv_norm));
      const double costheta3mu = pow(costheta, DMUL(3., F.mu));
      const double R_eq = pow_one_third(DDIV(DMUL(3., M), DMUL(FOUR_PI, avg)));
      const double vesc = __dsqrt_rn(DDIV(DMUL(DMUL(2., F.G), M), R_eq));
      const double K = DMUL(DDIV(DDIV(DMUL(DMUL(3., F.k), m_1), FOUR_PI), rho_12), costheta3mu);
      const double m_check =
          DMUL(K, DSUB(DMUL(pow(DDIV(DMUL(F.C1, dv_norm), vesc), DMUL(3., F.mu)), rho_12_3nu), 1.));
      double m_tilde = DSUB(M, m_check);
      const double m_tilde_2 = DDIV(m_check, (double)F.N_tilde);
      const double t = ap.t;
      double v_cm[3], r_cm[3];
      v_cm[0] = DDIV(DADD(DMUL(m_2, vx_a), DMUL(m_1, vx_b)), M);
      v_cm[1] = DDIV(DADD(DMUL(m_2, vy_a), DMUL(m_1, vy_b)), M);
      v_cm[2] = DDIV(DADD(DMUL(m_2, vz_a), DMUL(m_1, vz_b)), M);
      r_cm[0] = DDIV(DADD(DMUL(m_2, xa), DMUL(m_1, xb)), M);
      r_cm[1] = DDIV(DADD(DMUL(m_2, ya), DMUL(m_1, yb)), M);
      r_cm[2] = DDIV(DADD(DMUL(m_2, za), DMUL(m_1, zb)), M);
      if (rec) {
            rec[5] = dv_norm;
            rec[6] = dr_dot_dv;
            rec[7] = m_tilde;
      }
      out.nids = 0;

      if (m_check <= DMUL(F.merging_threshold, M)) {  // merger
            d_merge(S, a, b, ap, F.one_only, F.mesh_bool, nullptr);
            S.scal[S_FMERGE] += 1;
            out.outcome = 0;
            return;
      }
      if (m_tilde < DMUL(0.1, M)) {  // super-catastrophic: only the largest fragment stays
            m_tilde = DMUL(DMUL(0.1, M), pow(DDIV(DMUL(DDIV(1.0, 0.9), m_check), M), -1.5));
            S.vx[a] = v_cm[0]; S.vy[a] = v_cm[1]; S.vz[a] = v_cm[2];
            S.x[a] = DSUB(r_cm[0], DMUL(t, v_cm[0]));
            S.y[a] = DSUB(r_cm[1], DMUL(t, v_cm[1]));
            S.z[a] = DSUB(r_cm[2], DMUL(t, v_cm[2]));
            S.m[a] = m_tilde;
            S.R[a] = pow_one_third(DDIV(DMUL(3., m_tilde), DMUL(FOUR_PI, avg)));
            S.scal[S_NEEDCOM] = 1;
            d_lose(S, b, F.mesh_bool);
            S.did[a] = F.one_only;
            S.scal[S_FSUPER] += 1;
            double discarded = DSUB(M, m_tilde);
            if (m_tilde < DDIV(F.fragment_threshold, 4.)) {
                  d_lose(S, a, F.mesh_bool);
                  discarded = M;
            }
            if (F.central_mass_bool) F.cm[6] = DADD(F.cm[6], discarded);
            if (rec) rec[7] = m_tilde;
            out.outcome = 1;
            return;
      }
      if (m_tilde_2 < F.fragment_threshold && m_check <= m_tilde) {  // partial: the tail is one body
            const double vks = DMUL(DDIV(DMUL(DDIV(vesc, stigma), DADD(m_check, K)), m_check),
                                    DSUB(1.0, pow(DDIV(K, DADD(K, m_check)), stigma)));
            if (vks < vesc) {
                  atomicOr(err, ERR_FRAGMENT);
                  out.outcome = -1;
                  return;
            }
            const double in_front_of = DDIV(vks, R);
            double rk[3] = {-dx, -dy, -dz};
            double vk[3];
            for (int d = 0; d < 3; d++) vk[d] = DMUL(in_front_of, rk[d]);
            const double R_tilde = pow_one_third(DDIV(DMUL(3.0, m_tilde), DMUL(FOUR_PI, avg)));
            const double R_check = pow_one_third(DDIV(DMUL(3.0, m_check), DMUL(FOUR_PI, avg)));
            const double R_tilde12 = DADD(R_tilde, R_check);
            const double dr_norm = __dsqrt_rn(DADD(DADD(DMUL(rk[0], rk[0]), DMUL(rk[1], rk[1])), DMUL(rk[2], rk[2])));
            const double sc = DDIV(R_tilde12, dr_norm);
            for (int d = 0; d < 3; d++) rk[d] = DMUL(rk[d], sc);
            const double f = DDIV(m_check, M);
            double rt[3], vt[3];
            for (int d = 0; d < 3; d++) {
                  rt[d] = DSUB(r_cm[d], DMUL(f, rk[d]));
                  vt[d] = DSUB(v_cm[d], DMUL(f, vk[d]));
            }
            S.x[a] = DSUB(rt[0], DMUL(t, vt[0]));
            S.y[a] = DSUB(rt[1], DMUL(t, vt[1]));
            S.z[a] = DSUB(rt[2], DMUL(t, vt[2]));
            S.vx[a] = vt[0]; S.vy[a] = vt[1]; S.vz[a] = vt[2];
            S.m[a] = m_tilde;
            S.R[a] = R_tilde;
            S.x[b] = DSUB(DADD(rt[0], rk[0]), DMUL(t, DADD(vt[0], vk[0])));
            S.y[b] = DSUB(DADD(rt[1], rk[1]), DMUL(t, DADD(vt[1], vk[1])));
            S.z[b] = DSUB(DADD(rt[2], rk[2]), DMUL(t, DADD(vt[2], vk[2])));
            S.vx[b] = DADD(vt[0], vk[0]); S.vy[b] = DADD(vt[1], vk[1]); S.vz[b] = DADD(vt[2], vk[2]);
            S.m[b] = m_check;
            S.R[b] = R_check;
            S.did[a] = F.one_only;
            S.did[b] = F.one_only;
            S.scal[S_FHALF] += 1;
            out.outcome = 2;
            out.nids = 2;
            out.ids[0] = a;
            out.ids[1] = b;
            return;
      }
      // full fragmentation: N_tilde tail fragments on the (p, q) lattice
      const double R_tilde = pow_one_third(DDIV(DMUL(3.0, m_tilde), DMUL(FOUR_PI, avg)));
      const double R_tilde_2 = pow_one_third(DDIV(DMUL(3.0, m_tilde_2), DMUL(FOUR_PI, avg)));
      const double R_tilde12 = DADD(R_tilde, R_tilde_2);
      double dr[3] = {-dx, -dy, -dz};
      const double dv[3] = {-dvx, -dvy, -dvz};
      const double dr_norm = __dsqrt_rn(DADD(DADD(DMUL(dr[0], dr[0]), DMUL(dr[1], dr[1])), DMUL(dr[2], dr[2])));
      const double sc = DDIV(R_tilde12, dr_norm);
      for (int d = 0; d < 3; d++) dr[d] = DMUL(dr[d], sc);
      double dxv[3], u[3], v[3];
      d_cross(dr[0], dr[1], dr[2], dv[0], dv[1], dv[2], dxv);
      const double dxv_norm =
          __dsqrt_rn(DADD(DADD(DMUL(dxv[0], dxv[0]), DMUL(dxv[1], dxv[1])), DMUL(dxv[2], dxv[2])));
      if (dxv_norm > 1.0e-5) {  // oblique impact
            for (int d = 0; d < 3; d++) v[d] = DDIV(dxv[d], dxv_norm);
      } else {  // nearly frontal: any unit vector orthogonal to dr (maximum(), src/structure.c:1090)
            const double f0 = fabs(dr[0]), f1 = fabs(dr[1]), f2 = fabs(dr[2]);
            int mm = f0 >= f1 ? 0 : 1;
            const double mx = f0 >= f1 ? f0 : f1;
            if (!(mx >= f2)) mm = 2;
            const int i0 = mm, i1 = mm == 0 ? 1 : 0, i2 = mm == 2 ? 1 : 2;
            const double num = DADD(dr[i1], dr[i2]);
            const double w = DDIV(1.0, __dsqrt_rn(DADD(2.0, DDIV(DMUL(num, num), DMUL(dr[i0], dr[i0])))));
            v[i1] = w;
            v[i2] = w;
            v[i0] = DDIV(DMUL(-w, num), dr[i0]);
      }
      double vxd[3];
      d_cross(v[0], v[1], v[2], dr[0], dr[1], dr[2], vxd);
      for (int d = 0; d < 3; d++) u[d] = DDIV(vxd[d], R_tilde12);
      // momentum correction: sums of the tail offsets in lattice order
      double corr[6] = {0., 0., 0., 0., 0., 0.};
      {
            int n = 0;
            bool ok = true;
            for (int p = F.pq[0]; p <= F.pq[1]; p++)
                  for (int q = F.pq[2]; q <= F.pq[3]; q++) {
                        double rk[3], vk[3];
                        ok &= d_tail(n, p, q, dr, u, v, R_tilde_2, R_tilde12, m_tilde_2, K, m_check, stigma, vesc,
                                     rk, vk);
                        for (int d = 0; d < 3; d++) {
                              corr[d] = DADD(corr[d], rk[d]);
                              corr[3 + d] = DADD(corr[3 + d], vk[d]);
                        }
                        n++;
                  }
            if (!ok) {
                  atomicOr(err, ERR_FRAGMENT);
                  out.outcome = -1;
                  return;
            }
      }
      const double f = DDIV(m_tilde_2, M);
      double rt[3], vt[3];
      for (int d = 0; d < 3; d++) {
            rt[d] = DSUB(r_cm[d], DMUL(f, corr[d]));
            vt[d] = DSUB(v_cm[d], DMUL(f, corr[3 + d]));
      }
      out.ids[0] = a;
      for (int n = 1; n <= F.N_tilde; n++) {
            const int id = d_free_index(S, F.at_end, F.n_max, err);
            if (id < 0) {
                  out.outcome = -1;
                  return;
            }
            out.ids[n] = id;
      }
      out.nids = F.N_tilde + 1;
      d_lose(S, b, F.mesh_bool);
      for (int n = 0; n <= F.N_tilde; n++) S.did[out.ids[n]] = F.one_only;
      S.x[a] = DSUB(rt[0], DMUL(t, vt[0]));
      S.y[a] = DSUB(rt[1], DMUL(t, vt[1]));
      S.z[a] = DSUB(rt[2], DMUL(t, vt[2]));
      S.vx[a] = vt[0]; S.vy[a] = vt[1]; S.vz[a] = vt[2];
      S.m[a] = m_tilde;
      S.R[a] = R_tilde;
      int n = 0;
      for (int p = F.pq[0]; p <= F.pq[1]; p++)
            for (int q = F.pq[2]; q <= F.pq[3]; q++) {
                  double rk[3], vk[3];
                  d_tail(n, p, q, dr, u, v, R_tilde_2, R_tilde12, m_tilde_2, K, m_check, stigma, vesc, rk, vk);
                  const int id = out.ids[n + 1];
                  S.x[id] = DSUB(DADD(rt[0], rk[0]), DMUL(t, DADD(vt[0], vk[0])));
                  S.y[id] = DSUB(DADD(rt[1], rk[1]), DMUL(t, DADD(vt[1], vk[1])));
                  S.z[id] = DSUB(DADD(rt[2], rk[2]), DMUL(t, DADD(vt[2], vk[2])));
                  S.vx[id] = DADD(vt[0], vk[0]);
                  S.vy[id] = DADD(vt[1], vk[1]);
                  S.vz[id] = DADD(vt[2], vk[2]);
                  S.m[id] = m_tilde_2;
                  S.R[id] = R_tilde_2;
                  n++;
            }
      S.scal[S_FFULL] += 1;
      out.outcome = 3;
}

// FragArgs from the library parameters; false when N_tilde and the lattice
// do not agree (N_tilde = (p_max - p_min + 1)(q_max - q_min + 1), src/parameters.h:307-309).
inline bool make_frag_args(const Ctx &c, FragArgs &F)
{
      const ncgpu_params &P = c.P;
      F.N_tilde = P.par_N_tilde;
      for (int j = 0; j < 4; j++) F.pq[j] = P.par_pq_min_max[j];
      F.mu = P.par_mu_parameter;
      F.nu = P.par_nu_parameter;
      F.C1 = P.par_C1_parameter;
      F.k = P.par_k_parameter;
      F.merging_threshold = P.par_merging_threshold;
      F.fragment_threshold = P.par_fragment_threshold;
      F.G = P.par_G;
      F.central_mass_bool = P.par_central_mass_bool;
      F.at_end = P.par_mesh_bool && !c.force_naive;
      F.mesh_bool = P.par_mesh_bool;
      F.one_only = P.par_one_collision_only_bool;
      F.n_max = c.n_max;
      F.cm = c.cm;
      const long np = (long)F.pq[1] - F.pq[0] + 1, nq = (long)F.pq[3] - F.pq[2] + 1;
      return F.N_tilde >= 1 && F.N_tilde <= NCGPU_MAX_N_TILDE && np > 0 && nq > 0 && np * nq == F.N_tilde;
}

}  // namespace ncg
