// Total energy of the device state, a diagnostic with no counterpart in the
// reference (which has no energy output): the drift of this quantity over a
// run measures the integrator and force error of a gravity mode.
//
//   E = sum_k m_k |v_k|^2 / 2 + M |V|^2 / 2                  (kinetic)
//     - sum_k G M m_k / |r_k - R|                            (central body)
//     + sum_k m_k G M R_u^2 J2 (3 dz^2 - r^2) / (2 r^5)       (J2, r = r_k - R)
//     - sum_{k<p} G m_k m_p / sqrt(|r_k - r_p|^2 + eps^2)    (mutual)
//
// with eps = softening_parameter (R_k + R_p), the softening of the force
// (src/physics.c:187).  FP64 throughout; one block per 256 existing bodies
// sums its bodies' terms (each mutual pair counted from both sides, halved),
// block partials are added in block order, so the result is deterministic.
#include "common.cuh"

namespace ncg {
namespace {

constexpr int EB = 256;

__global__ void __launch_bounds__(EB) k_energy_part(BodyView bv, const int *__restrict__ cidx, int n,
                                                    const double *__restrict__ cm, double G, double sp, int central,
                                                    int mutual, J2Arg j2, double *__restrict__ part)
{
      __shared__ double sx[EB], sy[EB], sz[EB], sm[EB], sr[EB];
      __shared__ double red[3][EB];
      const int q = blockIdx.x * EB + threadIdx.x;
      const bool live = q < n;
      const int k = live ? cidx[q] : 0;
      const long s = bv.stride;
      const double x = bv.x[k * s], y = bv.y[k * s], z = bv.z[k * s], m = live ? bv.m[k * s] : 0.;
      const double R = bv.R[k * s];
      double kin = 0., pc = 0., pm = 0.;
      if (live) {
            const double vx = bv.vx[k * s], vy = bv.vy[k * s], vz = bv.vz[k * s];
            kin = 0.5 * m * (vx * vx + vy * vy + vz * vz);
            if (central) {
                  const double dx = x - cm[0], dy = y - cm[1], dz = z - cm[2];
                  const double r2 = dx * dx + dy * dy + dz * dz, r = sqrt(r2);
                  pc = -G * cm[6] * m / r;
                  if (j2.on)  // the potential whose gradient is the force of src/physics.c:149-160
                        pc += m * G * cm[6] * j2.R * j2.R * j2.J2 * (3. * dz * dz - r2) / (2. * r2 * r2 * r);
            }
      }
      for (int t0 = 0; mutual && t0 < n; t0 += EB) {
            __syncthreads();
            const int j = t0 + threadIdx.x;
            if (j < n) {
                  const int p = cidx[j];
                  sx[threadIdx.x] = bv.x[p * s];
                  sy[threadIdx.x] = bv.y[p * s];
                  sz[threadIdx.x] = bv.z[p * s];
                  sm[threadIdx.x] = bv.m[p * s];
                  sr[threadIdx.x] = bv.R[p * s];
            }
            __syncthreads();
            const int cnt = min(EB, n - t0);
            if (!live) continue;
            double acc = 0.;
            for (int jj = 0; jj < cnt; jj++) {
                  if (t0 + jj == q) continue;
                  const double dx = x - sx[jj], dy = y - sy[jj], dz = z - sz[jj];
                  const double e = sp * (R + sr[jj]);
                  acc += sm[jj] / sqrt(dx * dx + dy * dy + dz * dz + e * e);
            }
            pm += acc;
      }
      red[0][threadIdx.x] = kin;
      red[1][threadIdx.x] = pc;
      red[2][threadIdx.x] = live ? -0.5 * G * m * pm : 0.;
      __syncthreads();
      for (int o = EB / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o)
                  for (int d = 0; d < 3; d++) red[d][threadIdx.x] += red[d][threadIdx.x + o];
            __syncthreads();
      }
      if (threadIdx.x < 3) part[blockIdx.x * 3 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_energy_final(const double *__restrict__ part, int nparts, const double *__restrict__ cm,
                               int central, double *__restrict__ out)
{
      if (threadIdx.x != 0) return;
      double e[3] = {0., 0., 0.};
      for (int b = 0; b < nparts; b++)
            for (int d = 0; d < 3; d++) e[d] += part[3 * b + d];
      if (central) e[0] += 0.5 * cm[6] * (cm[3] * cm[3] + cm[4] * cm[4] + cm[5] * cm[5]);
      out[0] = e[0] + e[1] + e[2];
      out[1] = e[0];
      out[2] = e[1];
      out[3] = e[2];
}

}  // namespace
}  // namespace ncg

using namespace ncg;

extern "C" int ncgpu_energy(double *energy)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      if (!energy) return NCGPU_E_ARG;
      cudaStream_t st = c.s;
      int n = 0;
      NCG_TRY(compact_existing(c.ex, c.largest_id, &n, st));
      const int nb = n > 0 ? (n + EB - 1) / EB : 0;
      NCG_TRY(ensure_partial((size_t)3 * (nb > 0 ? nb : 1) + 4));
      BodyView bv{c.x, c.y, c.z, c.vx, c.vy, c.vz, c.m, c.R, 1, c.ex};
      double cmh[9] = {0., 0., 0., 0., 0., 0., 1., 0., 0.};  // the J2 term needs the central mass
      if (c.P.par_J2_bool) NCG_TRY(state_cm_host(cmh));
      if (nb > 0) {
            k_energy_part<<<nb, EB, 0, st>>>(bv, c.cidx, n, c.cm, c.P.par_G, c.P.par_softening_parameter,
                                             c.P.par_central_mass_bool, c.P.par_mutual_bool, j2_arg(c.P, cmh[6], c.j2),
                                             c.partial);
            NCG_LAUNCHED();
      }
      double *out = c.partial + 3 * (size_t)nb;
      k_energy_final<<<1, 32, 0, st>>>(c.partial, nb, c.cm, c.P.par_central_mass_bool, out);
      NCG_LAUNCHED();
      NCG_CK(cudaMemcpyAsync(energy, out, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaStreamSynchronize(st));
      return NCGPU_OK;
}
