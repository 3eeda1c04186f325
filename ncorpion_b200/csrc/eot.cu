// End of timestep on the device-resident state (src/rk4.c:130-404, the
// parts the hot path needs): dumping into the central mass or beyond the
// outer threshold, barycentre reduction, did_collide reset and tidy_up.
// Order-dependent updates (the central mass absorbing dumped bodies, the
// sequential momentum sums of total_momentum, src/structure.c:1193-1227) run
// in slot order on one thread per sum, so results match the reference bit for
// bit; the O(N) scans around them are parallel.
#include <algorithm>
#include "common.cuh"
#include "physics.cuh"

namespace ncg {

DevState dev_state();
int sync_scalars();
int kick_state();
int drift_state();
int collide_brute_state(bool defer);
int mesh_reset_state();
int mesh_pass(double gam, int test, bool defer);
void mesh_counts_finish(const int *h);
int three_largest_state(int *idx);

namespace {

// flag[j] = 1 (inside disruption_threshold, central mass on), 2 (beyond
// high_dumping_threshold), 0 otherwise; counts the bodies that stay.
__global__ void k_eot_flag(const DevState S, int lid, const double *__restrict__ cm, int central, double dis,
                           double high, int *__restrict__ flag)
{
      int j = blockIdx.x * blockDim.x + threadIdx.x;
      int f = 0;
      bool stays = false;
      if (j <= lid && S.ex[j]) {
            double XX = central ? cm[0] : 0., YY = central ? cm[1] : 0., ZZ = central ? cm[2] : 0.;
            double DX = DSUB(S.x[j], XX), DY = DSUB(S.y[j], YY), DZ = DSUB(S.z[j], ZZ);
            double r2 = DADD(DADD(DMUL(DX, DX), DMUL(DY, DY)), DMUL(DZ, DZ));
            if (r2 < DMUL(dis, dis) && central) f = 1;
            else if (r2 > DMUL(high, high)) f = 2;
            else stays = true;
      }
      if (j <= lid) flag[j] = f;
      // counts summed per block: one atomic on each counter per block instead of
      // one per body (atomics on one address are serialised at the L2)
      __shared__ int cnt[2];
      if (threadIdx.x < 2) cnt[threadIdx.x] = 0;
      __syncthreads();
      const unsigned m = __ballot_sync(0xffffffffu, f != 0), ms = __ballot_sync(0xffffffffu, stays);
      if ((threadIdx.x & 31) == 0) {
            if (m) atomicAdd(&cnt[0], __popc(m));
            if (ms) atomicAdd(&cnt[1], __popc(ms));
      }
      __syncthreads();
      if (threadIdx.x == 0) {
            if (cnt[0]) atomicAdd(S.scal + S_NFLAG, cnt[0]);
            if (cnt[1]) atomicAdd(S.scal + S_HM, cnt[1]);
      }
}

// The flagged bodies, in slot order (list from an order-preserving compaction).
__global__ void k_eot_dump(const DevState S, const int *__restrict__ list, int n, const int *__restrict__ flag,
                           double *cm, int mesh_bool)
{
      if (threadIdx.x != 0) return;
      for (int q = 0; q < n; q++) {
            int j = list[q];
            if (flag[j] == 1) {
                  double m = S.m[j];
                  double X = S.x[j], Y = S.y[j], Z = S.z[j], vX = S.vx[j], vY = S.vy[j], vZ = S.vz[j];
                  cm[6] = DADD(cm[6], m);
                  double M = cm[6];
                  double f = DDIV(DSUB(M, m), M);
                  for (int d = 0; d < 6; d++) cm[d] = DMUL(cm[d], f);
                  cm[0] = DADD(cm[0], DDIV(DMUL(m, X), M));
                  cm[1] = DADD(cm[1], DDIV(DMUL(m, Y), M));
                  cm[2] = DADD(cm[2], DDIV(DMUL(m, Z), M));
                  cm[3] = DADD(cm[3], DDIV(DMUL(m, vX), M));
                  cm[4] = DADD(cm[4], DDIV(DMUL(m, vY), M));
                  cm[5] = DADD(cm[5], DDIV(DMUL(m, vZ), M));
                  d_lose(S, j, mesh_bool);
            } else {
                  d_lose(S, j, mesh_bool);
                  S.scal[S_NEEDCOM] = 1;
            }
      }
}

// total_momentum: lane d < 6 sums component d, lane 6 the mass, in slot order.
// total_momentum's terms in slot order: m_j x_j, m_j y_j, ... m_j vz_j and
// m_j (7 arrays of n), so the sums below read them coalesced.
__global__ void k_momentum_terms(const DevState S, const int *__restrict__ list, int n, double *__restrict__ terms)
{
      int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q >= n) return;
      int j = list[q];
      double m = S.m[j];
      terms[q] = DMUL(m, S.x[j]);
      terms[(size_t)n + q] = DMUL(m, S.y[j]);
      terms[2 * (size_t)n + q] = DMUL(m, S.z[j]);
      terms[3 * (size_t)n + q] = DMUL(m, S.vx[j]);
      terms[4 * (size_t)n + q] = DMUL(m, S.vy[j]);
      terms[5 * (size_t)n + q] = DMUL(m, S.vz[j]);
      terms[6 * (size_t)n + q] = m;
}

// The central body's share, which starts every sum (src/structure.c:1202-1210).
__device__ __forceinline__ double momentum_init(int d, const double *cm, int central)
{
      const double M = central ? cm[6] : 0.;
      return d == 6 ? M : DMUL(M, central ? cm[d] : 0.);
}

// total_momentum (src/structure.c:1193-1227) in the reference's order: one
// CTA (one warp) per component sums its n terms sequentially (FP64, no
// reassociation, warp_chain_sum) into tot[0..6]; k_momentum_div divides.
__global__ void __launch_bounds__(32) k_momentum_chains(const double *__restrict__ terms, int n,
                                                        const double *__restrict__ cm, int central,
                                                        double *__restrict__ tot)
{
      __shared__ __align__(16) double stage[CHN];
      const int w = blockIdx.x;
      const double s = warp_chain_sum(terms + (size_t)w * n, n, momentum_init(w, cm, central), stage);
      if (threadIdx.x == 0) tot[w] = s;
}

__global__ void k_momentum_div(const double *__restrict__ tot, double *__restrict__ com)
{
      if (threadIdx.x < 6) com[threadIdx.x] = DDIV(tot[threadIdx.x], tot[6]);
}

// The same sums as a deterministic two-level parallel reduction (non-exact
// gravity modes): block b adds a fixed slice, the fold adds the slices in order.
constexpr int MPB = 256;
__global__ void __launch_bounds__(MPB) k_momentum_part(const double *__restrict__ terms, int n,
                                                       double *__restrict__ part)
{
      __shared__ double sh[7][MPB / 32];
      double s[7] = {0., 0., 0., 0., 0., 0., 0.};
      for (int q = blockIdx.x * MPB + threadIdx.x; q < n; q += gridDim.x * MPB)
            for (int d = 0; d < 7; d++) s[d] += terms[(size_t)d * n + q];
      const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
      for (int d = 0; d < 7; d++) {
            double v = s[d];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) sh[d][wp] = v;
      }
      __syncthreads();
      if (threadIdx.x < 7) {
            double v = 0.;
            for (int q = 0; q < MPB / 32; q++) v += sh[threadIdx.x][q];
            part[blockIdx.x * 7 + threadIdx.x] = v;
      }
}

__global__ void k_momentum_fold(const double *__restrict__ part, int nparts, const double *__restrict__ cm,
                                int central, double *__restrict__ com)
{
      __shared__ double tot[7];
      const int d = threadIdx.x;
      if (d < 7) {
            double s = 0.;
            for (int b = 0; b < nparts; b++) s += part[7 * b + d];
            tot[d] = momentum_init(d, cm, central) + s;
      }
      __syncthreads();
      if (d < 6) com[d] = tot[d] / tot[6];
}

__global__ void k_sub_com(const DevState S, int lid, const double *__restrict__ com, double *cm, int central)
{
      int j = blockIdx.x * blockDim.x + threadIdx.x;
      if (j == 0 && central)
            for (int d = 0; d < 6; d++) cm[d] = DSUB(cm[d], com[d]);
      if (j <= lid && S.ex[j]) {
            S.x[j] = DSUB(S.x[j], com[0]); S.y[j] = DSUB(S.y[j], com[1]); S.z[j] = DSUB(S.z[j], com[2]);
            S.vx[j] = DSUB(S.vx[j], com[3]); S.vy[j] = DSUB(S.vy[j], com[4]); S.vz[j] = DSUB(S.vz[j], com[5]);
      }
}

// tidy_up (src/structure.c:881-911): existing bodies moved to slots 0..n-1
// in order (gather through a staging copy).
__global__ void k_tidy_gather(const DevState S, const int *__restrict__ list, int n, double *__restrict__ tmp,
                              long N)
{
      int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q >= n) return;
      int j = list[q];
      tmp[q] = S.x[j]; tmp[N + q] = S.y[j]; tmp[2 * N + q] = S.z[j];
      tmp[3 * N + q] = S.vx[j]; tmp[4 * N + q] = S.vy[j]; tmp[5 * N + q] = S.vz[j];
      tmp[6 * N + q] = S.m[j]; tmp[7 * N + q] = S.R[j];
}

__global__ void k_tidy_scatter(const DevState S, int n, int lid, const double *__restrict__ tmp, long N)
{
      int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q < n) {
            S.x[q] = tmp[q]; S.y[q] = tmp[N + q]; S.z[q] = tmp[2 * N + q];
            S.vx[q] = tmp[3 * N + q]; S.vy[q] = tmp[4 * N + q]; S.vz[q] = tmp[5 * N + q];
            S.m[q] = tmp[6 * N + q]; S.R[q] = tmp[7 * N + q];
      }
      if (q <= lid) S.ex[q] = q < n ? 1 : 0;
      if (q == 0) {
            S.scal[S_LID] = n - 1;
            S.scal[S_NFREE] = 0;
      }
}

}  // namespace

// total_momentum (src/structure.c:1193-1227) of the state into com[0..5]
// (device; com[8..14] scratch): the position and velocity of the barycentre,
// sequential FP64 sums in slot order (exact) or a parallel reduction.
int total_momentum_dev(bool exact, double *com)
{
      Ctx &c = ctx();
      cudaStream_t st = c.s;
      const ncgpu_params &P = c.P;
      DevState S = dev_state();
      int n = 0;
      NCG_TRY(compact_existing(c.ex, c.largest_id, &n, st));
      if (n > 0) {
            NCG_TRY(ensure_partial((size_t)7 * n + 7 * 148));
            double *terms = c.partial;
            k_momentum_terms<<<(n + 255) / 256, 256, 0, st>>>(S, c.cidx, n, terms);
            NCG_LAUNCHED();
            if (exact) {
                  k_momentum_chains<<<7, 32, 0, st>>>(terms, n, c.cm, P.par_central_mass_bool, com + 8);
                  NCG_LAUNCHED();
                  k_momentum_div<<<1, 32, 0, st>>>(com + 8, com);
                  NCG_LAUNCHED();
            } else {
                  const int np = std::min(148, (n + MPB - 1) / MPB);
                  double *part = terms + (size_t)7 * n;
                  k_momentum_part<<<np, MPB, 0, st>>>(terms, n, part);
                  NCG_LAUNCHED();
                  k_momentum_fold<<<1, 32, 0, st>>>(part, np, c.cm, P.par_central_mass_bool, com);
                  NCG_LAUNCHED();
            }
      } else {
            k_momentum_fold<<<1, 32, 0, st>>>(c.red + 3584, 0, c.cm, P.par_central_mass_bool, com);
            NCG_LAUNCHED();
      }
      return NCGPU_OK;
}

int eot_state(int *hm_out)
{
      Ctx &c = ctx();
      cudaStream_t st = c.s;
      const ncgpu_params &P = c.P;
      const int lid = c.largest_id;
      c.eot_lid = lid;  // largest_id before tidy_up, which end_of_timestep prints
      DevState S = dev_state();
      NCG_CK(cudaMemsetAsync(c.scal + S_HM, 0, 2 * sizeof(int), st));  // HM, NFLAG
      const int nb = lid >= 0 ? (lid + 256) / 256 : 1;
      int *flag = c.exs;
      k_eot_flag<<<nb, 256, 0, st>>>(S, lid, c.cm, P.par_central_mass_bool, P.par_disruption_threshold,
                                     P.par_high_dumping_threshold, flag);
      NCG_LAUNCHED();
      int h[S_COUNT];
      unsigned e = 0;  // the step's device errors come back with the counts
      NCG_CK(cudaMemcpyAsync(h, c.scal, sizeof h, cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaMemcpyAsync(&e, c.err, sizeof e, cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaStreamSynchronize(st));
      if (e) NCG_TRY(check_err_word());
      c.n_events = h[S_NEV];  // (a collision pass of this step may have left these to us)
      c.collision_count = h[S_CCOUNT];
      mesh_counts_finish(h);
      const int hm = h[S_HM];
      const bool changed = h[S_NFLAG] > 0 || hm < 9 * lid / 10;  // dumping or tidy_up change the scalars
      if (h[S_NFLAG] > 0) {
            int nf = 0;
            NCG_TRY(compact_existing(flag, lid, &nf, st));
            k_eot_dump<<<1, 32, 0, st>>>(S, c.cidx, nf, flag, c.cm, P.par_mesh_bool);
            NCG_LAUNCHED();
            NCG_CK(cudaMemcpyAsync(h, c.scal, sizeof h, cudaMemcpyDeviceToHost, st));
            NCG_CK(cudaStreamSynchronize(st));
      }
      c.com_reduced = 0;
      if (h[S_NEEDCOM] && P.par_reduce_to_COM_bool) {
            double *com = c.red + 3072;
            NCG_TRY(total_momentum_dev(P.par_gravity_mode == NCGPU_GRAVITY_EXACT, com));
            c.com_reduced = 1;
            k_sub_com<<<nb, 256, 0, st>>>(S, lid, com, c.cm, P.par_central_mass_bool);
            NCG_LAUNCHED();
            NCG_CK(cudaMemsetAsync(c.scal + S_NEEDCOM, 0, sizeof(int), st));
      }
      if (P.par_mesh_bool) NCG_TRY(mesh_reset_state());  // hash table cleared (src/rk4.c:356-364)
      if (P.par_collision_bool && (P.par_one_collision_only_bool || P.par_collision_type == NCGPU_COLLISION_FRAGMENTATION))
            NCG_CK(cudaMemsetAsync(c.did, 0, sizeof(int) * (size_t)(lid + 1 > 0 ? lid + 1 : 1), st));
      if (hm < 9 * lid / 10) {
            int n = 0;
            NCG_TRY(compact_existing(c.ex, lid, &n, st));
            if (n > 0) {
                  k_tidy_gather<<<(n + 255) / 256, 256, 0, st>>>(S, c.cidx, n, c.aos, c.n_max);
                  NCG_LAUNCHED();
            }
            k_tidy_scatter<<<nb, 256, 0, st>>>(S, n, lid, c.aos, c.n_max);
            NCG_LAUNCHED();
      }
      if (changed) NCG_TRY(sync_scalars());
      if (P.par_J2_bool && P.par_J2 == 0.) NCG_TRY(refresh_j2());  // src/rk4.c:459-463
      if (hm_out) *hm_out = hm;
      return NCGPU_OK;
}

}  // namespace ncg

using namespace ncg;

// end_of_timestep's barycentre printout (src/rk4.c:202-222, 333): zeros right
// after an end of step that reduced the barycentre, else the state's
// total_momentum now (exact sums).
extern "C" int ncgpu_total_momentum(double *com)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      if (!com) return NCGPU_E_ARG;
      if (c.com_reduced) {  // end_of_timestep zeroes the vector it subtracted (src/rk4.c:219)
            for (int d = 0; d < 6; d++) com[d] = 0.;
            return NCGPU_OK;
      }
      double *d = c.red + 3072;
      NCG_TRY(total_momentum_dev(true, d));
      NCG_CK(cudaMemcpyAsync(com, d, 6 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
      NCG_CK(cudaStreamSynchronize(c.s));
      return NCGPU_OK;
}

extern "C" int ncgpu_get_largest_id(int *largest_id, int *before_tidy)
{
      Ctx &c = ctx();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      if (!largest_id) return NCGPU_E_ARG;
      *largest_id = c.largest_id;
      if (before_tidy) *before_tidy = c.eot_lid;
      return NCGPU_OK;
}

extern "C" int ncgpu_end_of_timestep(int *how_many_moonlets)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      return eot_state(how_many_moonlets);
}

extern "C" int ncgpu_step_brute_force(int *how_many_moonlets)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      NCG_TRY(kick_state());
      if (c.P.par_collision_bool) NCG_TRY(collide_brute_state(true));  // its counts come back with the end of step's
      NCG_TRY(drift_state());
      return eot_state(how_many_moonlets);
}

// One iteration of integration_mesh's loop (src/rk4.c:760-790) with mesh size
// gam; *total_neighbours is the pass's count for the host's gamma update.
extern "C" int ncgpu_step_mesh(double gam, int *how_many_moonlets, long *total_neighbours)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      if (!(gam > 0.)) return NCGPU_E_ARG;
      long tn = 0;
      if (c.P.par_collision_bool) {
            if (c.force_naive) {
                  NCG_TRY(collide_brute_state(false));
            } else {
                  NCG_TRY(three_largest_state(nullptr));
                  NCG_TRY(mesh_pass(gam, 1, true));  // its counts come back with the end of step's
            }
      }
      NCG_TRY(drift_state());
      if (!c.P.par_collision_bool && !c.force_naive) {
            NCG_TRY(three_largest_state(nullptr));
            NCG_TRY(mesh_pass(gam, 0, false));
            tn = c.total_neighbours;
      }
      NCG_TRY(kick_state());
      const int st = eot_state(how_many_moonlets);
      if (c.P.par_collision_bool && !c.force_naive) tn = c.total_neighbours;  // (set by the end of step's read)
      if (total_neighbours) *total_neighbours = tn;
      return st;
}
