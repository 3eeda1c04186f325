// Brute-force collision search with in-place resolution: the device
// replacement of brute_force (src/collision.c:425-456).
//
// The reference sweeps i = 0..largest_id (bound frozen at entry), j = i+1..
// largest_id (bound re-read), and resolves every colliding pair on the spot,
// so later predicates see the updated bodies.  On the GPU:
//
//   1. k_bf_hits      every pair (i < j) of the entry state is tested in FP64
//                     (exact reference arithmetic) by a tiled sweep; colliding
//                     pairs are appended through a warp-aggregated atomic
//                     counter.
//   2. sort           hits ordered by (i, j) with two stable radix passes.
//   3. k_bf_events    one CTA replays the sweep order: the next event is the
//                     smallest (i, j) after the last one that either is an
//                     entry-state hit between two untouched bodies, or involves
//                     a body an earlier event modified and collides with the
//                     current state (those pairs are re-tested in parallel by
//                     the CTA).  Events are resolved one by one with the
//                     reference's arithmetic, so state and event order match.
#include "common.cuh"
#include "physics.cuh"

namespace ncg {

namespace {

constexpr int BT = 128;          // bodies per tile of the hit sweep
constexpr int EVT = 1024;        // threads of the event kernel

__device__ __forceinline__ void append_hit(bool hit, int i, int j, int *hi, int *hj, int *count, int cap,
                                           unsigned *err)
{
      unsigned m = __ballot_sync(0xffffffffu, hit);
      if (!m) return;
      int lane = threadIdx.x & 31;
      int leader = __ffs(m) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(count, __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (hit) {
            int pos = base + __popc(m & ((1u << lane) - 1u));
            if (pos < cap) {
                  hi[pos] = i;
                  hj[pos] = j;
            } else {
                  atomicOr(err, ERR_CAPACITY);
            }
      }
}

// One CTA per (i tile, j tile) with j tile >= i tile; thread = body i.
__global__ void __launch_bounds__(BT) k_bf_hits(DevState S, int lid, double dt, int *hi, int *hj, int cap,
                                                unsigned *err)
{
      // tile (ti, tj), tj >= ti: body i of the thread against the tile's bodies j
      // staged in shared memory (closest_approach's test on the same values)
      __shared__ double sj[7][BT];
      __shared__ int sv[BT];
      const int ti = blockIdx.y, tj = blockIdx.x;
      if (tj < ti) return;
      const int i = ti * BT + threadIdx.x;
      const bool vi = i <= lid && S.ex[i] && !S.did[i];
      double xi = 0., yi = 0., zi = 0., vxi = 0., vyi = 0., vzi = 0., Ri = 0.;
      if (vi) {
            xi = S.x[i]; yi = S.y[i]; zi = S.z[i]; vxi = S.vx[i]; vyi = S.vy[i]; vzi = S.vz[i]; Ri = S.R[i];
      }
      const int j0 = tj * BT;
      const int jn = min(BT, lid + 1 - j0);
      if ((int)threadIdx.x < jn) {
            const int j = j0 + threadIdx.x;
            sj[0][threadIdx.x] = S.x[j]; sj[1][threadIdx.x] = S.y[j]; sj[2][threadIdx.x] = S.z[j];
            sj[3][threadIdx.x] = S.vx[j]; sj[4][threadIdx.x] = S.vy[j]; sj[5][threadIdx.x] = S.vz[j];
            sj[6][threadIdx.x] = S.R[j];
            sv[threadIdx.x] = S.ex[j] && !S.did[j];
      }
      __syncthreads();
      for (int jj = 0; jj < jn; ++jj) {
            const int j = j0 + jj;
            bool hit = false;
            double t;
            if (vi && j > i && sv[jj])
                  hit = d_contact(xi, yi, zi, vxi, vyi, vzi, Ri, sj[0][jj], sj[1][jj], sj[2][jj], sj[3][jj], sj[4][jj],
                                  sj[5][jj], sj[6][jj], dt, &t);
            append_hit(hit, i, j, hi, hj, S.scal + S_NHITS, cap, err);
      }
}

__global__ void k_gather_int(const int *__restrict__ src, const int *__restrict__ idx, int n, int *__restrict__ dst)
{
      int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q < n) dst[q] = src[idx[q]];
}

__global__ void k_iota(int *v, int n)
{
      int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q < n) v[q] = q;
}

__device__ __forceinline__ unsigned long long pkey(int p, int q)
{
      return ((unsigned long long)(unsigned)p << 32) | (unsigned)q;
}

struct EvArgs {
      int lid0;                 // i-loop bound frozen at entry (current_largest_id)
      double dt;
      int type;                 // collision_treatment type
      double f_inelastic;
      int one_only;
      int mesh_bool;
      int ev_cap;
      int dcap;
      FragArgs frag;            // fragmentation constants (type 3)
};

// collision_treatment(a, b, type) with the device state; records the event.
__device__ void d_treat(const DevState &S, int a, int b, const EvArgs &E, int *ev, double *evrec,
                        unsigned char *dirty, int *dlist, unsigned *err)
{
      Approach ap;
      d_approach(S, a, b, E.dt, &ap);  // true for every event the sweep selects
      double m_a = S.m[a], m_b = S.m[b];
      int A = m_a > m_b ? a : b, B = m_a > m_b ? b : a;
      int ne = S.scal[S_NEV];
      double *rec = nullptr;
      if (ne < E.ev_cap) {
            ev[3 * ne] = a;
            ev[3 * ne + 1] = b;
            ev[3 * ne + 2] = E.type;
            rec = evrec + (size_t)EVREC * ne;
            rec[0] = ap.t;
            rec[1] = S.m[A];
            rec[2] = S.m[B];
            rec[3] = S.R[A];
            rec[4] = S.R[B];
      } else {
            atomicOr(err, ERR_CAPACITY);
      }
      S.scal[S_NEV] = ne + 1;
      if (E.type == NCGPU_COLLISION_ELASTIC || E.type == NCGPU_COLLISION_INELASTIC) {
            d_impulse(S, A, B, E.type == NCGPU_COLLISION_ELASTIC ? 2.0 : E.f_inelastic, ap, rec);
            S.did[a] = E.one_only;
            S.did[b] = E.one_only;
      } else if (E.type == NCGPU_COLLISION_MERGER) {
            d_merge(S, A, B, ap, E.one_only, E.mesh_bool, rec);
      }
      FragOut fo;
      fo.nids = 0;
      if (E.type == NCGPU_COLLISION_FRAGMENTATION) d_fragment(S, A, B, ap, E.frag, rec, fo, err);
      S.scal[S_CCOUNT] += 1;
      // mark the bodies the resolution touched (new tail fragments included);
      // the ones that still exist are re-tested against the rest of the sweep
      int nd = S.scal[S_NDIRTY];
      const int nw = 2 + (fo.nids > 1 ? fo.nids - 1 : 0);
      for (int w = 0; w < nw; w++) {
            int k = w == 0 ? A : w == 1 ? B : fo.ids[w - 1];
            if (!dirty[k]) {
                  dirty[k] = 1;
                  if (nd < E.dcap) dlist[nd++] = k;
                  else atomicOr(err, ERR_CAPACITY);
            }
      }
      S.scal[S_NDIRTY] = nd;
}

__global__ void __launch_bounds__(EVT) k_bf_events(DevState S, const int *__restrict__ hi, const int *__restrict__ hj,
                                                   EvArgs E, int *ev, double *evrec, unsigned char *dirty, int *dlist,
                                                   unsigned *err)
{
      __shared__ unsigned long long best;
      __shared__ unsigned long long candA;
      __shared__ int hp_s;
      const unsigned long long INF = ~0ull;
      const int nh = min(S.scal[S_NHITS], (int)0x7fffffff);
      unsigned long long cur = 0;  // key of the last event; (0, 0) is never a pair
      if (threadIdx.x == 0) hp_s = 0;
      __syncthreads();
      // keys strictly increase from one event to the next, so the loop ends;
      // the bound only guards against a corrupted state
      for (int iter = 0;; ++iter) {
            if (iter > (1 << 26)) {
                  if (threadIdx.x == 0) atomicOr(err, ERR_TIMEOUT);
                  break;
            }
            if (threadIdx.x == 0) {
                  int hp = hp_s;
                  while (hp < nh && (pkey(hi[hp], hj[hp]) <= cur || dirty[hi[hp]] || dirty[hj[hp]])) hp++;
                  hp_s = hp;
                  candA = hp < nh ? pkey(hi[hp], hj[hp]) : INF;
                  best = candA;
            }
            __syncthreads();
            const int nd = S.scal[S_NDIRTY];
            const int lidnow = S.scal[S_LID];
            for (int di = 0; di < nd; di++) {
                  const int d = dlist[di];
                  if (!S.ex[d] || S.did[d]) continue;
                  for (int x = threadIdx.x; x <= lidnow; x += EVT) {
                        if (x == d) continue;
                        int p = min(d, x), q = max(d, x);
                        unsigned long long key = pkey(p, q);
                        if (key <= cur || key >= best || p > E.lid0) continue;
                        if (!S.ex[x] || S.did[x]) continue;
                        if (d_approach(S, p, q, E.dt, nullptr)) atomicMin(&best, key);
                  }
            }
            __syncthreads();
            const unsigned long long nxt = best;
            if (nxt == INF) break;
            if (threadIdx.x == 0) {
                  int p = (int)(nxt >> 32), q = (int)(nxt & 0xffffffffu);
                  d_treat(S, p, q, E, ev, evrec, dirty, dlist, err);
            }
            cur = nxt;
            __syncthreads();
      }
}

__global__ void k_clear_dirty(unsigned char *dirty, const int *dlist, const int *scal)
{
      int n = scal[S_NDIRTY];
      for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) dirty[dlist[k]] = 0;
}

}  // namespace

DevState dev_state()
{
      Ctx &c = ctx();
      return DevState{c.x, c.y, c.z, c.vx, c.vy, c.vz, c.m, c.R, c.ex, c.did, c.free_idx, c.scal};
}

static int bits_for(int maxval)
{
      int b = 1;
      while (b < 31 && (1 << b) <= maxval) b++;
      return b;
}

// Sorts the n hits (hi, hj) by (i, j) into (out_i, out_j).
static int sort_hits(int n, int *out_i, int *out_j, int lid, cudaStream_t st)
{
      Ctx &c = ctx();
      if (n == 0) return NCGPU_OK;
      int nb = (n + 255) / 256;
      int bits = bits_for(lid);
      NCG_CK(cudaMemcpyAsync(c.keys, c.hj, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, st));
      k_iota<<<nb, 256, 0, st>>>(c.vals, n);
      NCG_LAUNCHED();
      NCG_TRY(radix_sort_pairs(c.keys, c.vals, n, bits, st));  // by j
      k_gather_int<<<nb, 256, 0, st>>>(c.hi, c.vals, n, (int *)c.keys);
      NCG_LAUNCHED();
      NCG_TRY(radix_sort_pairs(c.keys, c.vals, n, bits, st));  // stable by i
      k_gather_int<<<nb, 256, 0, st>>>(c.hi, c.vals, n, out_i);
      NCG_LAUNCHED();
      k_gather_int<<<nb, 256, 0, st>>>(c.hj, c.vals, n, out_j);
      NCG_LAUNCHED();
      return NCGPU_OK;
}

// Reads back the scalars a sweep changed and the device error word.
int sync_scalars() { int h[S_COUNT]; return sync_scalars_h(h); }

// sync_scalars, also handing the device scalars to the caller (h: S_COUNT ints)
int sync_scalars_h(int *h)
{
      Ctx &c = ctx();
      unsigned e = 0;  // the device scalars and the error word behind one synchronisation
      NCG_CK(cudaMemcpyAsync(h, c.scal, sizeof(int) * S_COUNT, cudaMemcpyDeviceToHost, c.s));
      NCG_CK(cudaMemcpyAsync(&e, c.err, sizeof e, cudaMemcpyDeviceToHost, c.s));
      NCG_CK(cudaStreamSynchronize(c.s));
      c.largest_id = h[S_LID];
      c.n_events = h[S_NEV];
      c.collision_count = h[S_CCOUNT];
      if (!e) return NCGPU_OK;
      return check_err_word();  // reads, clears and maps the recorded error
}

// defer: leave the scalars' read-back to the caller's next synchronisation
// (the end of step's), for the collision types that append no body (largest_id
// cannot change).
int collide_brute_state(bool defer)
{
      Ctx &c = ctx();
      cudaStream_t st = c.s;
      const int lid = c.largest_id;
      if (lid < 1) {
            NCG_CK(cudaMemsetAsync(c.scal + S_NEV, 0, sizeof(int), st));
            return sync_scalars();
      }
      // S_NHITS, S_NEV, S_NDIRTY = 0
      NCG_CK(cudaMemsetAsync(c.scal + S_NHITS, 0, 2 * sizeof(int), st));
      NCG_CK(cudaMemsetAsync(c.scal + S_NDIRTY, 0, sizeof(int), st));
      DevState S = dev_state();
      const int nt = (lid + BT) / BT;
      dim3 grid(nt, nt);
      k_bf_hits<<<grid, BT, 0, st>>>(S, lid, c.dt, c.hi, c.hj, c.hit_cap, c.err);
      NCG_LAUNCHED();
      int nh = 0;
      NCG_CK(cudaMemcpyAsync(&nh, c.scal + S_NHITS, sizeof(int), cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaStreamSynchronize(st));
      if (nh > c.hit_cap) return NCGPU_E_CAPACITY;
      int *si = c.hi + c.hit_cap / 2, *sj = c.hj + c.hit_cap / 2;  // sorted hits (upper halves)
      if (nh > c.hit_cap / 2) return NCGPU_E_CAPACITY;
      NCG_TRY(sort_hits(nh, si, sj, lid, st));
      EvArgs E{lid, c.dt, c.P.par_collision_type, c.P.par_collision_parameter, c.P.par_one_collision_only_bool,
               c.P.par_mesh_bool, c.ev_cap, c.n_max, FragArgs{}};
      if (E.type == NCGPU_COLLISION_FRAGMENTATION && !make_frag_args(c, E.frag)) return NCGPU_E_ARG;
      k_bf_events<<<1, EVT, 0, st>>>(S, si, sj, E, c.ev, c.evrec, c.dirty, c.dlist, c.err);
      NCG_LAUNCHED();
      k_clear_dirty<<<32, 256, 0, st>>>(c.dirty, c.dlist, c.scal);
      NCG_LAUNCHED();
      if (defer && E.type != NCGPU_COLLISION_FRAGMENTATION) return NCGPU_OK;
      return sync_scalars();
}

}  // namespace ncg

using namespace ncg;

extern "C" int ncgpu_fragment_counts(int *counts)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      if (!counts) return NCGPU_E_ARG;
      NCG_CK(cudaMemcpyAsync(counts, c.scal + S_FMERGE, 4 * sizeof(int), cudaMemcpyDeviceToHost, c.s));
      NCG_CK(cudaStreamSynchronize(c.s));
      return NCGPU_OK;
}

extern "C" int ncgpu_collide_brute(int *n_events)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      NCG_TRY(collide_brute_state(false));
      if (n_events) *n_events = c.n_events;
      return NCGPU_OK;
}

extern "C" int ncgpu_get_events(struct ncgpu_event *out, double *records, int cap, int *n)
{
      Ctx &c = ctx();
      if (!c.inited) return NCGPU_E_STATE;
      if (!n) return NCGPU_E_ARG;
      int k = c.n_events < cap ? c.n_events : cap;
      if (k > c.ev_cap) k = c.ev_cap;
      if (k > 0 && out)
            NCG_CK(cudaMemcpyAsync(out, c.ev, sizeof(int) * 3 * (size_t)k, cudaMemcpyDeviceToHost, c.s));
      if (k > 0 && records)
            NCG_CK(cudaMemcpyAsync(records, c.evrec, sizeof(double) * EVREC * (size_t)k, cudaMemcpyDeviceToHost, c.s));
      NCG_CK(cudaStreamSynchronize(c.s));
      *n = c.n_events;
      return NCGPU_OK;
}

namespace ncg {
namespace {
__global__ void k_pow_third(const double *__restrict__ x, double *__restrict__ out, int n)
{
      int i = blockIdx.x * blockDim.x + threadIdx.x;
      if (i < n) out[i] = pow_one_third(x[i]);
}
}  // namespace
}  // namespace ncg

extern "C" int ncgpu_probe_pow_third(const double *x, double *out, int n)
{
      if (!x || !out || n <= 0) return NCGPU_E_ARG;
      double *d = nullptr;
      NCG_CK(cudaMalloc(&d, 2 * sizeof(double) * (size_t)n));
      NCG_CK(cudaMemcpy(d, x, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice));
      k_pow_third<<<(n + 255) / 256, 256>>>(d, d + n, n);
      NCG_LAUNCHED();
      NCG_CK(cudaMemcpy(out, d + n, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost));
      NCG_CK(cudaFree(d));
      return NCGPU_OK;
}
