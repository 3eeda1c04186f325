// Tides raised on the central body, constant time lag model: the device
// replacement of tides (src/physics.c:496-542), which kick calls after the
// vector field (src/rk4.c:88-90).
//
// For every existing body j, in slot order, with the state before the kick
// (X = r_j - r_CM, v relative to the central body and advanced half a kick
// with the vector field's accelerations), the reference computes
//   K = 3 k2 G R^5 m / r^10,  S = 1 / (1 + m/M)
//   a = S K (r^2 X + Delta_t (2 (r.v) X + r^2 (v + r x Omega)))
// subtracts a from the body's acceleration, adds a m / M to CM_acc and then
//   SideralOmega += timestep m / (moi M R^2) (X a_y - Y a_x) / S,
// and the next body's r x Omega uses the new SideralOmega.  That recurrence is
// sequential, but a body's increment is usually far below half an ulp of
// SideralOmega, so that the sum leaves it unchanged.  The work is split in three:
//   k_tides_prep   one thread per body: everything that does not depend on
//                  SideralOmega (the z component entirely), as 13 doubles a body,
//                  and then, speculatively, the body's step with the rotation the
//                  kick starts from; the first body whose step would change the
//                  rotation is recorded (every step before it used the right
//                  value, so its results are final);
//   k_tides_chain  one warp, from that body on (nothing when no body changes
//                  the rotation): lane 0 runs the recurrence in slot order (11
//                  dependent FP64 operations and a division a body) while the
//                  warp stages the next records through shared memory;
//   k_tides_apply  one thread per body: the accelerations and CM_acc terms,
//                  then CM_acc's sums from the vector field's value (sequential
//                  in the exact gravity mode, a parallel reduction otherwise).
// Every operation is the reference's, in its order, with IEEE rounding.
#include "common.cuh"
#include "physics.cuh"

namespace ncg {

int compact_existing(const int *ex, int largest_id, int *n_host, cudaStream_t st);
DevState dev_state();

namespace {

constexpr int TREC = 13;  // doubles per record
// record: X, Y, vX, vY, r2, r2*X, r2*Y, (2 rv)*X, (2 rv)*Y, S*K, timestep m/(moi M R R), S, 1/S
enum { RX, RY, RVX, RVY, RR2, RR2X, RR2Y, RTX, RTY, RSK, RCQ, RS, RYS };

// One body's step of the recurrence: its (a_x, a_y) with rotation W, and the
// rotation after it (src/physics.c:523-539).
__device__ __forceinline__ double tide_step(const double *r, double W, double Dt, double &aX, double &aY)
{
      const double oX = DMUL(r[RY], W);   // r_x_OmX =  Y*SideralOmega
      const double oY = DMUL(-r[RX], W);  // r_x_OmY = -X*SideralOmega
      aX = DMUL(r[RSK], DADD(r[RR2X], DMUL(Dt, DADD(r[RTX], DMUL(r[RR2], DADD(r[RVX], oX))))));
      aY = DMUL(r[RSK], DADD(r[RR2Y], DMUL(Dt, DADD(r[RTY], DMUL(r[RR2], DADD(r[RVY], oY))))));
      return DADD(W, div_by_recip(DMUL(r[RCQ], DSUB(DMUL(r[RX], aY), DMUL(r[RY], aX))), r[RS], r[RYS]));
}

__global__ void k_tides_prep(DevState S, const int *__restrict__ cidx, int n, const double *__restrict__ cm,
                             const double *__restrict__ cm_acc, const double *__restrict__ ax,
                             const double *__restrict__ ay, double *__restrict__ az, double dt, double A, double Dt,
                             double moi, double R, double *__restrict__ rec, double *__restrict__ terms,
                             double *__restrict__ aout, int *__restrict__ first)
{
      const int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q >= n) return;
      const int k = cidx[q];
      const double M = cm[6];
      const double X = DSUB(S.x[k], cm[0]), Y = DSUB(S.y[k], cm[1]), Z = DSUB(S.z[k], cm[2]);
      const double h = DMUL(0.5, dt);
      const double vX = DADD(DSUB(S.vx[k], cm[3]), DMUL(h, DSUB(ax[k], cm_acc[0])));
      const double vY = DADD(DSUB(S.vy[k], cm[4]), DMUL(h, DSUB(ay[k], cm_acc[1])));
      const double vZ = DADD(DSUB(S.vz[k], cm[5]), DMUL(h, DSUB(az[k], cm_acc[2])));
      const double m = S.m[k];
      const double r2 = DADD(DADD(DMUL(X, X), DMUL(Y, Y)), DMUL(Z, Z));
      const double r10 = DMUL(DMUL(DMUL(DMUL(r2, r2), r2), r2), r2);
      const double rv = DADD(DADD(DMUL(X, vX), DMUL(Y, vY)), DMUL(Z, vZ));
      const double K = DDIV(DMUL(A, m), r10);
      const double Sf = DDIV(1., DADD(1., DDIV(m, M)));
      const double SK = DMUL(Sf, K);
      const double tr = DMUL(2., rv);
      // aZ = S*K*(r2*Z + Delta_t*(2.*rv*Z + r2*vZ)): no SideralOmega in it
      const double aZ = DMUL(SK, DADD(DMUL(r2, Z), DMUL(Dt, DADD(DMUL(tr, Z), DMUL(r2, vZ)))));
      az[k] = DSUB(az[k], aZ);
      terms[2 * (size_t)n + q] = DDIV(DMUL(aZ, m), M);
      double *r = rec + (size_t)TREC * q;
      r[RX] = X;
      r[RY] = Y;
      r[RVX] = vX;
      r[RVY] = vY;
      r[RR2] = r2;
      r[RR2X] = DMUL(r2, X);
      r[RR2Y] = DMUL(r2, Y);
      r[RTX] = DMUL(tr, X);
      r[RTY] = DMUL(tr, Y);
      r[RSK] = SK;
      r[RCQ] = DDIV(DMUL(dt, m), DMUL(DMUL(DMUL(moi, M), R), R));
      r[RS] = Sf;
      r[RYS] = __drcp_rn(Sf);
      // the step with the rotation the kick starts from: final for every body
      // before the first one whose step changes the rotation
      const double W0 = cm[8];
      double aX, aY;
      if (tide_step(r, W0, Dt, aX, aY) != W0) atomicMin(first, q);
      aout[2 * (size_t)q] = aX;
      aout[2 * (size_t)q + 1] = aY;
}

constexpr int TBK = 64;                 // records staged per block
constexpr int TPER = TBK * TREC / 32;   // doubles each lane stages per block

// The SideralOmega recurrence in slot order (one warp) from the first body
// whose step changes the rotation (none: nothing to do); writes (a_x, a_y) of
// those bodies to aout and the final SideralOmega to cm[8].
__global__ void __launch_bounds__(32) k_tides_chain(const double *__restrict__ rec, int n, double Dt, double *cm,
                                                    double *__restrict__ aout, const int *__restrict__ first)
{
      __shared__ __align__(16) double st[TBK * TREC];
      __shared__ double ob[2 * TBK];
      const int lane = threadIdx.x;
      const int q0 = *first;
      if (q0 >= n) return;
      const long total = (long)n * TREC;
      double v[TPER];
#pragma unroll
      for (int u = 0; u < TPER; u++) {
            const long i = (long)q0 * TREC + (long)u * 32 + lane;
            v[u] = i < total ? rec[i] : 0.;
      }
      double W = cm[8];
      for (int base = q0; base < n; base += TBK) {
#pragma unroll
            for (int u = 0; u < TPER; u++) st[u * 32 + lane] = v[u];
            __syncwarp();
#pragma unroll
            for (int u = 0; u < TPER; u++) {  // the next block, in flight during the recurrence
                  const long i = (long)(base + TBK) * TREC + (long)u * 32 + lane;
                  v[u] = i < total ? rec[i] : 0.;
            }
            const int cnt = min(TBK, n - base);
            if (lane == 0) {
                  for (int q = 0; q < cnt; q++) {
                        double aX, aY;
                        W = tide_step(st + q * TREC, W, Dt, aX, aY);
                        ob[2 * q] = aX;
                        ob[2 * q + 1] = aY;
                  }
            }
            __syncwarp();
            for (int i = lane; i < 2 * cnt; i += 32) aout[2 * (size_t)base + i] = ob[i];
            __syncwarp();
      }
      if (lane == 0) cm[8] = W;
}

__global__ void k_tides_apply(DevState S, const int *__restrict__ cidx, int n, const double *__restrict__ cm,
                              const double *__restrict__ aout, double *__restrict__ ax, double *__restrict__ ay,
                              double *__restrict__ terms)
{
      const int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q >= n) return;
      const int k = cidx[q];
      const double aX = aout[2 * (size_t)q], aY = aout[2 * (size_t)q + 1];
      const double m = S.m[k], M = cm[6];
      ax[k] = DSUB(ax[k], aX);
      ay[k] = DSUB(ay[k], aY);
      terms[q] = DDIV(DMUL(aX, m), M);
      terms[(size_t)n + q] = DDIV(DMUL(aY, m), M);
}

}  // namespace

int tides_state(double *d_acc, long bs, double *d_cm_acc)
{
      Ctx &c = ctx();
      const ncgpu_params &P = c.P;
      cudaStream_t st = c.s;
      int n = 0;
      NCG_TRY(compact_existing(c.ex, c.largest_id, &n, st));
      if (n == 0) return NCGPU_OK;
      NCG_TRY(ensure_partial((size_t)(TREC + 2 + 3) * n + 1));
      double *rec = c.partial, *aout = rec + (size_t)TREC * n, *terms = aout + 2 * (size_t)n;
      int *first = (int *)(terms + 3 * (size_t)n);  // first body whose step changes the rotation
      NCG_CK(cudaMemsetAsync(first, 0x7f, sizeof(int), st));
      const double R = P.par_R_unit;
      const double R5 = R * R * R * R * R;
      const double A = 3. * P.par_k2 * P.par_G * R5;  // src/physics.c:505-506
      double *ax = d_acc, *ay = d_acc + bs, *az = d_acc + 2 * bs;
      DevState S = dev_state();
      const int nb = (n + 255) / 256;
      k_tides_prep<<<nb, 256, 0, st>>>(S, c.cidx, n, c.cm, d_cm_acc, ax, ay, az, c.dt, A, P.par_Delta_t,
                                       P.par_dimensionless_moi, R, rec, terms, aout, first);
      NCG_LAUNCHED();
      k_tides_chain<<<1, 32, 0, st>>>(rec, n, P.par_Delta_t, c.cm, aout, first);
      NCG_LAUNCHED();
      k_tides_apply<<<nb, 256, 0, st>>>(S, c.cidx, n, c.cm, aout, ax, ay, terms);
      NCG_LAUNCHED();
      // CM_acc += a m / M: in slot order (exact mode), or a parallel sum
      if (P.par_gravity_mode == NCGPU_GRAVITY_EXACT) return seq_sum3(terms, n, d_cm_acc, d_cm_acc, st);
      return par_sum3(terms, n, d_cm_acc, d_cm_acc, st);
}

}  // namespace ncg
