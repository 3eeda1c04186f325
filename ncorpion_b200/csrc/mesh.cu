// Mesh collision search: the device replacement of mesh() and
// get_neighbours_mesh() (src/collision.c:175-417, src/physics.c:1094-1118).
//
// The reference walks bodies k = 0..largest_id; a small body (R <= gam) first
// collects every body already in the 27 cells around its own cell, then
// inserts itself into its cell; the collected ids are popped in the order
// cell slot l = 26..0, ascending index within a cell (the LIFO of
// src/structure.c:712-841 reversed), each popped pair is tested by
// closest_approach in FP64 and either resolved on the spot or appended to
// pairs[].  Cells are identified by the reference's linear index
// i + j*d + k*d^2 (d = collision_cube_cells, i = d/2 + 1 + floor(X/gam)), so
// the neighbour aliasing of that index at the cube's x and y edges is kept.
//
// On the GPU:
//   k_mesh_keys     cell index per inserted body (-1 outside the cube)
//   radix sort      (cell, index) pairs; a dense cell -> first-position table
//                   (the analogue of the reference's (d+2)^3 hash table) gives
//                   O(1) access to a cell's bodies, in ascending index order
//   k_mesh_count    candidates per body = bodies of lower index in its 27 cells
//   scan            positions of every body's list in the global pop order
//   k_mesh_write    candidates (k, p) written in pop order; the FP64 predicate
//                   of the entry state marks hits
//   k_mesh_events   one CTA replays the hits in order (mesh_events.cu)
#include "common.cuh"
#include "physics.cuh"

namespace ncg {

namespace {

constexpr unsigned NOKEY = 0xffffffffu;

// linear cell index of a body, -1 outside the cube (src/collision.c:192-202)
__device__ __forceinline__ long long d_cell(double X, double Y, double Z, double gam, double half, int d)
{
      if (fabs(X) > half || fabs(Y) > half || fabs(Z) > half) return -1;
      long long i = d / 2 + 1 + (int)floor(DDIV(X, gam));
      long long j = d / 2 + 1 + (int)floor(DDIV(Y, gam));
      long long k = d / 2 + 1 + (int)floor(DDIV(Z, gam));
      return i + j * (long long)d + k * (long long)d * d;
}

// neighbour offset of cell slot l (l = 0 is (-1,-1,-1), x fastest)
__device__ __forceinline__ long long d_noff(int l, int d)
{
      int di = l % 3 - 1, dj = (l / 3) % 3 - 1, dk = l / 9 - 1;
      return di + dj * (long long)d + dk * (long long)d * d;
}

__global__ void k_mesh_keys(DevState S, int lid, double gam, double half, int d, int all_mode,
                            uint32_t *__restrict__ keys, int *__restrict__ vals, int *__restrict__ ckey,
                            int *__restrict__ nbig)
{
      int k = blockIdx.x * blockDim.x + threadIdx.x;
      if (k > lid) return;
      long long L = -1;
      if (S.ex[k]) {
            if (all_mode || S.R[k] <= gam) L = d_cell(S.x[k], S.y[k], S.z[k], gam, half, d);
            else atomicAdd(nbig, 1);
      }
      ckey[k] = (int)L;
      keys[k] = L >= 0 ? (uint32_t)L : NOKEY;
      vals[k] = k;
}

__global__ void k_cell_heads(const uint32_t *__restrict__ keys, int n, int2 *__restrict__ crange,
                             int *__restrict__ n_ins)
{
      int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q >= n) return;
      uint32_t key = keys[q];
      if (key == NOKEY) {
            if (q == 0 || keys[q - 1] != NOKEY) *n_ins = q;
            return;
      }
      if (q == 0 || keys[q - 1] != key) crange[key].x = q;
      if (keys[q + 1] != key) crange[key].y = q + 1;  // (keys[n] is the NOKEY sentinel)
      if (q == n - 1) *n_ins = n;
}

__global__ void k_cell_clear(const uint32_t *__restrict__ keys, int n, int2 *__restrict__ crange)
{
      int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q >= n) return;
      uint32_t key = keys[q];
      if (key != NOKEY && (q == 0 || keys[q - 1] != key)) crange[key] = make_int2(-1, -1);
}

// number of candidates of body k (lo <= k < hi): existing bodies of lower
// index in its 27 cells; 0 outside [lo, hi)
// Cell-ordered copy of the fields the pass reads: record q is body vals[q];
// pv[q] is vals[q] for an existing body, INT_MAX otherwise, so that "p < k and
// p exists" is one compact load (pv[q] < k).
__global__ void k_mesh_records(const DevState S, const int *__restrict__ vals, int n, MRec *__restrict__ rec,
                               int *__restrict__ pv)
{
      int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q >= n) return;
      const int b = vals[q];
      MRec r;
      r.x = S.x[b]; r.y = S.y[b]; r.z = S.z[b]; r.R = S.R[b];
      r.vx = S.vx[b]; r.vy = S.vy[b]; r.vz = S.vz[b];
      r.ex = S.ex[b];
      r.did = S.did[b];
      rec[q] = r;
      pv[q] = r.ex ? b : 0x7fffffff;
}

// The 27 neighbour cells as 9 rows of three consecutive linear indices
// (x - 1, x, x + 1): row r (0..8) has dy = r % 3 - 1, dz = r / 3 - 1, so the
// cell slots l = 26..0 of the pop order are the rows r = 8..0, each from x + 1
// down to x - 1.

__global__ void k_mesh_count(const int *__restrict__ pv, const int *__restrict__ ckey,
                             const int *__restrict__ vals, const int2 *__restrict__ crange, int lid, int lo, int hi,
                             int d, long long cap, int *__restrict__ cnt)
{
      // threads walk the bodies in cell order (vals = bodies sorted by cell), so
      // the threads of a warp share cells and partners
      const int t = blockIdx.x * blockDim.x + threadIdx.x;
      if (t > lid) return;
      const int k = vals[t];
      int L = (k >= lo && k < hi) ? ckey[k] : -1;
      int c = 0;
      if (L >= 0) {
            const long long dd = (long long)d * d;
            // a row's three cells are one contiguous range of the sorted bodies
#pragma unroll 1
            for (int r = 0; r < 9; ++r) {
                  const long long mid = d_row(L, r, d, dd);
                  int s, e;
                  if (!row_range(crange, mid, cap, &s, &e)) continue;
                  for (int q = s; q < e; ++q)
                        if (pv[q] < k) c++;  // (a body removed earlier in the pass is not pushed)
            }
      }
      cnt[k] = c;
}

// Candidates of body k in pop order; hit flag from the entry-state predicate.
//
// The warp's 32 bodies (consecutive in cell order) share the work: each lane
// queues the positions of every body in its 27 cells, in pop order (rows 8..0,
// cells x + 1 .. x - 1, each cell's bodies in ascending index), into shared
// memory; then the warp takes the queued entries 32 at a time, each lane one
// entry whatever list it belongs to.  An entry is a candidate when its body p
// has a lower index than the list's owner k and exists; its position is the
// owner's offset plus the number of the owner's candidates before it (a ballot
// over the round, plus a running count per owner), so the lists come out in
// the reference's order.  The candidates of one list are written by adjacent
// lanes (coalesced stores) and the FP64 predicates run with every lane busy.
// A lane whose queue is full walks again in the next round, queueing the
// entries after those already taken.
constexpr int MWW = 4;   // warps per block
constexpr int MWQ = 32;  // queued entries per lane and round

__global__ void __launch_bounds__(MWW * 32) k_mesh_write(const MRec *__restrict__ rec, const int *__restrict__ ckey,
                                                        const int *__restrict__ vals, const int *__restrict__ pv,
                                                        const int2 *__restrict__ crange,
                                                        const int *__restrict__ off, int lid, int lo, int hi, int d,
                                                        long long cap, double dt, int test, int *__restrict__ ck,
                                                        int *__restrict__ cp, unsigned char *__restrict__ cflag,
                                                        int *__restrict__ hitpos, int hit_cap, int *__restrict__ nhits,
                                                        long pair_cap, unsigned *err)
{
      __shared__ int qb[MWW][32 * MWQ];
      __shared__ unsigned char owner[MWW][32 * MWQ];
      __shared__ int pre[MWW][32], run[MWW][32], okk[MWW][32], opos[MWW][32];
      __shared__ MRec orec[MWW][32];  // the lists' owners' records
      const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
      const int t = blockIdx.x * blockDim.x + threadIdx.x;  // cell order, as k_mesh_count
      int k = -1, L = -1;
      if (t <= lid) {
            k = vals[t];
            if (k >= lo && k < hi) L = ckey[k];
      }
      bool dk = false;
      if (L >= 0) {
            const MRec rk = load_mrec(rec, t);
            orec[w][lane] = rk;
            dk = test && rk.did;
            opos[w][lane] = off[k];
      }
      okk[w][lane] = (L >= 0 ? k : -1) | (dk ? 0x80000000 : 0);
      run[w][lane] = 0;
      const long long dd = (long long)d * d;
      int skip = 0;
      bool more = L >= 0;
      while (__any_sync(0xffffffffu, more)) {
            int cnt = 0;
            if (more) {
                  int idx = 0;
#pragma unroll 1
                  for (int r = 8; r >= 0; --r) {
                        int2 cr[3];
                        row_cells(crange, d_row(L, r, d, dd), cap, cr);
#pragma unroll
                        for (int x = 2; x >= 0; --x) {  // cells mid + 1, mid, mid - 1
                              const int a = max(cr[x].x, cr[x].x + skip - idx), b = min(cr[x].y, cr[x].x + skip + MWQ - idx);
                              for (int q = a; q < b; ++q) qb[w][lane * MWQ + idx + (q - cr[x].x) - skip] = q;
                              if (cr[x].x >= 0) idx += cr[x].y - cr[x].x;
                        }
                  }
                  cnt = min(max(idx - skip, 0), MWQ);
                  more = idx > skip + MWQ;
            }
            int incl = cnt;
            for (int o = 1; o < 32; o <<= 1) {
                  const int u = __shfl_up_sync(0xffffffffu, incl, o);
                  if (lane >= o) incl += u;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            const int mine = incl - cnt;
            pre[w][lane] = mine;
            for (int j = 0; j < cnt; ++j) owner[w][mine + j] = (unsigned char)lane;
            __syncwarp();
            for (int f0 = 0; f0 < total; f0 += 32) {
                  const int fi = f0 + lane;
                  int o = -1, q = 0, p = 0, kk = -1;
                  bool cand = false;
                  if (fi < total) {
                        o = owner[w][fi];
                        q = qb[w][o * MWQ + fi - pre[w][o]];
                        kk = okk[w][o] & 0x7fffffff;
                        p = pv[q];
                        cand = p < kk;  // (a body removed earlier in the pass is not pushed)
                  }
                  const unsigned m = __ballot_sync(0xffffffffu, cand);
                  // this entry's list starts at lane a of the round (the lists are contiguous, in lane order)
                  const int a = o >= 0 ? max(pre[w][o] - f0, 0) : 0;
                  const unsigned below = (1u << lane) - 1u, from_a = ~((1u << a) - 1u);
                  const int nb = o >= 0 ? run[w][o] + __popc(m & below & from_a) : 0;
                  const int on = __shfl_down_sync(0xffffffffu, o, 1);
                  __syncwarp();
                  if (o >= 0 && (lane == 31 || on != o))  // the list's last entry in this round: its running count
                        run[w][o] += __popc(m & from_a & (lane == 31 ? 0xffffffffu : ((2u << lane) - 1u)));
                  if (cand) {
                        const long pos = (long)opos[w][o] + nb;
                        if (pos >= pair_cap) {
                              atomicOr(err, ERR_CAPACITY);
                        } else {
                              ck[pos] = kk;
                              cp[pos] = p;
                              unsigned char f = 0;
                              const MRec rp = load_mrec(rec, q);
                              if (test && !(okk[w][o] & 0x80000000) && !rp.did &&
                                  d_contact_rec(rp, orec[w][o], dt)) {  // closest_approach(p, k)
                                    f = 1;
                                    int h = atomicAdd(nhits, 1);
                                    if (h < hit_cap) hitpos[h] = (int)pos;
                                    else atomicOr(err, ERR_CAPACITY);
                              }
                              cflag[pos] = f;
                        }
                  }
                  __syncwarp();
            }
            skip += MWQ;
      }
}

}  // namespace

namespace {

// cflag bits
constexpr unsigned char F_HIT = 1, F_DROP = 2, F_MERGED = 4, F_SWAP = 8;
constexpr int MEV = 1024;       // threads of the event kernel

struct MeshEvArgs {
      int lid0, d, type, one_only, mesh_bool, ev_cap, dcap, occ_cap, nsorted;
      long long cell_cap;
      double dt, f_inelastic;
      int add_pairs;            // mutual_bool: pairs[] is kept
      long xpair_cap;
      FragArgs frag;            // fragmentation constants (type 3)
      int seg_hi;               // querying bodies of this replay: below seg_hi (candidate lists exist)
};

// Buffers of the fragmentation bookkeeping (see Ctx::evx).
struct MeshFragBufs {
      int *evx, *xpairs, *xhead, *fev;
};

// collision_treatment(p, k, type) at candidate position q (src/physics.c:1043).
// Candidate flags: F_SWAP = pairs[] gets (p, k) here instead of (k, p)
// (impulses; a partial fragmentation whose larger body is p); F_MERGED = no
// pair of its own here (merger, super-catastrophic, full fragmentation: the
// latter's tail pairs go to xpairs and are spliced in at this position).
__device__ void d_mesh_treat(const DevState &S, int p, int k, int q, const MeshEvArgs &E, int *ev, double *evrec,
                             unsigned char *cflag, const MeshFragBufs &X, unsigned *err, int *A_out, int *B_out)
{
      Approach ap;
      d_approach(S, p, k, E.dt, &ap);
      double m_a = S.m[p], m_b = S.m[k];
      int A = m_a > m_b ? p : k, B = m_a > m_b ? k : p;
      int ne = S.scal[S_NEV];
      double *rec = nullptr;
      int *ex_rec = nullptr;
      if (ne < E.ev_cap) {
            ev[3 * ne] = p;
            ev[3 * ne + 1] = k;
            ev[3 * ne + 2] = E.type;
            rec = evrec + (size_t)EVREC * ne;
            rec[0] = ap.t; rec[1] = S.m[A]; rec[2] = S.m[B]; rec[3] = S.R[A]; rec[4] = S.R[B];
            ex_rec = X.evx + (size_t)EVX * ne;
            ex_rec[0] = q;
            ex_rec[1] = S.scal[S_NXPAIRS];
            ex_rec[2] = 0;
            ex_rec[3] = -1;
            ex_rec[4] = A;
            ex_rec[5] = -1;
            ex_rec[6] = k;
            ex_rec[7] = p;
      } else {
            atomicOr(err, ERR_CAPACITY);
      }
      S.scal[S_NEV] = ne + 1;
      if (E.type == NCGPU_COLLISION_ELASTIC || E.type == NCGPU_COLLISION_INELASTIC) {
            d_impulse(S, A, B, E.type == NCGPU_COLLISION_ELASTIC ? 2.0 : E.f_inelastic, ap, rec);
            S.did[p] = E.one_only;
            S.did[k] = E.one_only;
            cflag[q] |= F_SWAP;   // pairs[] gets (p, k) at this position
      } else if (E.type == NCGPU_COLLISION_MERGER) {
            d_merge(S, A, B, ap, E.one_only, E.mesh_bool, rec);
            cflag[q] |= F_MERGED;  // no pair appended
            S.scal[S_NSKIP] += 1;
      } else {
            FragOut fo;
            d_fragment(S, A, B, ap, E.frag, rec, fo, err);
            if (fo.outcome == 2) {
                  if (A == p) cflag[q] |= F_SWAP;  // pairs[] gets (A, B)
            } else {
                  cflag[q] |= F_MERGED;
                  S.scal[S_NSKIP] += 1;
            }
            if (fo.outcome == 3) {
                  const int nt = fo.nids - 1;
                  int nx = S.scal[S_NXPAIRS];
                  const int cnt = E.add_pairs ? (nt + 1) * nt / 2 : 0;
                  if ((long)nx + cnt > E.xpair_cap) {
                        atomicOr(err, ERR_CAPACITY);
                  } else {
                        for (int a = 0; a <= nt && cnt; a++)
                              for (int b = 0; b < a; b++) {
                                    X.xpairs[2 * nx] = fo.ids[a];
                                    X.xpairs[2 * nx + 1] = fo.ids[b];
                                    nx++;
                              }
                        S.scal[S_NXPAIRS] = nx;
                  }
                  if (ex_rec) {
                        ex_rec[2] = cnt;
                        ex_rec[3] = fo.ids[1];  // the tail occupies fo.ids[1] .. fo.ids[1] + nt - 1
                        int nf = S.scal[S_NFEV];
                        X.fev[nf] = ne;
                        S.scal[S_NFEV] = nf + 1;
                        // chain of full fragmentations whose largest fragment is A
                        int h = X.xhead[A];
                        if (h < 0) {
                              X.xhead[A] = ne;
                        } else {
                              int guard = 0;
                              while (X.evx[(size_t)EVX * h + 5] >= 0 && ++guard < E.ev_cap) h = X.evx[(size_t)EVX * h + 5];
                              X.evx[(size_t)EVX * h + 5] = ne;
                        }
                  }
            }
      }
      S.scal[S_CCOUNT] += 1;
      *A_out = A;
      *B_out = B;
}

// One CTA.  hitpos: entry-state hits sorted by position.  Modified bodies get
// their later occurrences collected into a pool (own remaining pops, and the
// lists of later bodies in the 27 cells around them); those occurrences are
// re-tested against the current state after every event, the untouched hits
// are taken as they are, and the smallest position wins.
__global__ void __launch_bounds__(MEV) k_mesh_events(DevState S, const int *__restrict__ ck, const int *__restrict__ cp,
                                                     unsigned char *cflag, const int *__restrict__ off,
                                                     const int *__restrict__ ckey, const uint32_t *__restrict__ keys,
                                                     const int *__restrict__ vals, const int2 *__restrict__ crange,
                                                     const int *__restrict__ hitpos, int nh, MeshEvArgs E, int *ev,
                                                     double *evrec, unsigned char *dirty, int *occ, int *ndrop,
                                                     MeshFragBufs X, unsigned *err)
{
      __shared__ int best, hp_s, nocc, newb[2], newn, kq_s, q_s;
      if (threadIdx.x == 0) {
            hp_s = 0;
            nocc = 0;
      }
      __syncthreads();
      int cur = -1;
      for (int iter = 0;; ++iter) {
            if (iter > (1 << 26)) {
                  if (threadIdx.x == 0) atomicOr(err, ERR_TIMEOUT);
                  break;
            }
            if (threadIdx.x == 0) {
                  int hp = hp_s;
                  while (hp < nh) {
                        int q = hitpos[hp];
                        if (q > cur && !dirty[ck[q]] && !dirty[cp[q]] && !(cflag[q] & F_DROP)) break;
                        hp++;
                  }
                  hp_s = hp;
                  best = hp < nh ? hitpos[hp] : 0x7fffffff;
            }
            __syncthreads();
            const int no = nocc;
            for (int t = threadIdx.x; t < no; t += MEV) {
                  int q = occ[t];
                  if (q <= cur || q >= best || (cflag[q] & (F_DROP | F_MERGED | F_SWAP))) continue;
                  int k = ck[q], p = cp[q];
                  if (S.did[k] || S.did[p]) continue;
                  if (d_approach(S, p, k, E.dt, nullptr)) atomicMin(&best, q);
            }
            __syncthreads();
            const int q = best;
            if (q == 0x7fffffff) break;
            if (threadIdx.x == 0) {
                  int A, B;
                  int k = ck[q], p = cp[q];
                  d_mesh_treat(S, p, k, q, E, ev, evrec, cflag, X, err, &A, &B);
                  // dirty: 1 = modified (its later occurrences are re-tested), 2 = removed
                  // (its later occurrences are dropped).  A body already modified by an
                  // earlier event and removed by this one is processed again.
                  int nn = 0;
                  const int who[2] = {A, B};
                  for (int w = 0; w < 2; w++) {
                        const int x = who[w];
                        if (w == 1 && x == A) break;
                        const unsigned char want = S.ex[x] ? 1 : 2;
                        if (dirty[x] < want) {
                              dirty[x] = want;
                              newb[nn++] = x;
                        }
                  }
                  newn = nn;
                  kq_s = k;
                  q_s = q;
            }
            __syncthreads();
            // occurrences of the newly modified bodies after position q
            const int kq = kq_s, nn = newn;
            for (int w = 0; w < nn; ++w) {
                  const int x = newb[w];
                  const bool alive = S.ex[x];
                  // remaining pops of the querying body itself
                  if (x == kq && alive)
                        for (int r = q_s + 1 + threadIdx.x; r < off[kq + 1]; r += MEV) {
                              int o = atomicAdd(&nocc, 1);
                              if (o < E.occ_cap) occ[o] = r;
                              else atomicOr(err, ERR_CAPACITY);
                        }
                  // x in the lists of later bodies of its 27 cells
                  const int Lx = ckey[x];
                  if (Lx < 0) continue;
                  for (int l = threadIdx.x >> 5; l < 27; l += MEV / 32) {
                        long long cell = Lx + d_noff(l, E.d);
                        if (cell < 0 || cell >= E.cell_cap) continue;
                        int s = crange[cell].x;
                        if (s < 0) continue;
                        for (int qq = s + (threadIdx.x & 31); qq < E.nsorted && keys[qq] == (uint32_t)cell; qq += 32) {
                              int kk = vals[qq];
                              if (kk <= kq || kk >= E.seg_hi) continue;
                              for (int r = off[kk]; r < off[kk + 1]; ++r) {
                                    if (cp[r] != x) continue;
                                    if (alive) {
                                          int o = atomicAdd(&nocc, 1);
                                          if (o < E.occ_cap) occ[o] = r;
                                          else atomicOr(err, ERR_CAPACITY);
                                    } else {
                                          cflag[r] |= F_DROP;  // removed before kk's query: never pushed
                                    }
                              }
                        }
                  }
                  // a removed body does not query its own cells either
                  if (!alive && x > kq && x < E.seg_hi)
                        for (int r = off[x] + threadIdx.x; r < off[x + 1]; r += MEV) cflag[r] |= F_DROP;
            }
            cur = q;
            __syncthreads();
      }
}

// Number of dropped candidates (a candidate can be dropped by two removals).
__global__ void k_count_dropped(const unsigned char *__restrict__ cflag, int n, int *__restrict__ ndrop)
{
      int q = blockIdx.x * blockDim.x + threadIdx.x;
      int d = q < n && (cflag[q] & F_DROP) ? 1 : 0;
      d = __syncthreads_count(d);
      if (threadIdx.x == 0 && d) atomicAdd(ndrop, d);
}

// ---- bodies larger than the mesh size (src/collision.c:380-410) ----------

// The smallest slot k in [lo, lid] holding a body larger than the mesh size.
__global__ void k_next_big(const DevState S, int lo, int lid, double gam, int *__restrict__ out)
{
      int k = lo + blockIdx.x * blockDim.x + threadIdx.x;
      if (k <= lid && S.ex[k] && S.R[k] > gam) atomicMin(out, k);
}

// Cell keys for a pass resumed at slot lo: bodies below lo keep the cell they
// were inserted in; the others get the cell of their current position (or
// none: removed, larger than the mesh size, outside the cube).
__global__ void k_mesh_rekey(const DevState S, int lo, int lid, double gam, double half, int d,
                             uint32_t *__restrict__ keys, int *__restrict__ vals, int *__restrict__ ckey)
{
      int k = blockIdx.x * blockDim.x + threadIdx.x;
      if (k > lid) return;
      long long L;
      if (k < lo) {
            L = ckey[k];
      } else {
            L = -1;
            if (S.ex[k] && S.R[k] <= gam) L = d_cell(S.x[k], S.y[k], S.z[k], gam, half, d);
            ckey[k] = (int)L;
      }
      keys[k] = L >= 0 ? (uint32_t)L : NOKEY;
      vals[k] = k;
}

__global__ void k_add_base(int *__restrict__ off, int n, int base)
{
      int k = blockIdx.x * blockDim.x + threadIdx.x;
      if (k <= n) off[k] += base;
}

// The big-body branch of mesh() for body e at its turn, one CTA: every
// existing p != e with R_p < gam, or p > e, in ascending p up to the live
// largest_id (tail fragments made meanwhile are visited too), becomes the
// candidate (e, p) at positions base, base + 1, ...; collisions are resolved
// one at a time in p order against the current state.  *count gets the number
// of candidates written.
constexpr int BVT = 1024;
__global__ void __launch_bounds__(BVT) k_big_visit(DevState S, int e, double gam, int base, long cap, MeshEvArgs E,
                                                   int *__restrict__ ck, int *__restrict__ cp,
                                                   unsigned char *__restrict__ cflag, int *ev, double *evrec,
                                                   MeshFragBufs X, int *__restrict__ count, unsigned *err)
{
      __shared__ int ws[BVT / 32];
      __shared__ int s_lid, s_pos, s_first;
      const int t = threadIdx.x, lane = t & 31, w = t >> 5;
      if (t == 0) s_pos = base;
      int p0 = 0;
      for (int iter = 0;; ++iter) {
            if (iter > (1 << 24)) {
                  if (t == 0) atomicOr(err, ERR_TIMEOUT);
                  break;
            }
            __syncthreads();
            if (t == 0) s_lid = S.scal[S_LID];
            __syncthreads();
            const int lid = s_lid;
            if (p0 > lid) break;
            const int p = p0 + t;
            const bool qual = p <= lid && S.ex[p] && p != e && (S.R[p] < gam || p > e);
            // exclusive rank of this candidate within the chunk
            const unsigned bal = __ballot_sync(0xffffffffu, qual);
            int rank = __popc(bal & ((1u << lane) - 1u));
            if (lane == 0) ws[w] = __popc(bal);
            __syncthreads();
            if (w == 0) {
                  int v = ws[lane];
                  for (int o = 1; o < 32; o <<= 1) {
                        int u = __shfl_up_sync(0xffffffffu, v, o);
                        if (lane >= o) v += u;
                  }
                  ws[lane] = v;  // inclusive
            }
            __syncthreads();
            rank += w > 0 ? ws[w - 1] : 0;
            const int chunk = ws[BVT / 32 - 1];
            const long q = (long)s_pos + rank;
            if (qual) {
                  if (q < cap) {
                        ck[q] = e;
                        cp[q] = p;
                        cflag[q] = 0;
                  } else {
                        atomicOr(err, ERR_CAPACITY);
                  }
            }
            // collisions in p order: the first hit is resolved, the rest re-tested
            int from = p0;
            for (int r = 0; r <= BVT; ++r) {
                  const bool hit = qual && p >= from && q < cap && !S.did[e] && !S.did[p] &&
                                   d_approach(S, p, e, E.dt, nullptr);
                  if (t == 0) s_first = 0x7fffffff;
                  __syncthreads();
                  if (hit) atomicMin(&s_first, p);
                  __syncthreads();
                  const int ph = s_first;
                  if (ph == 0x7fffffff) break;
                  if (p == ph) {
                        int A, B;
                        d_mesh_treat(S, p, e, (int)q, E, ev, evrec, cflag, X, err, &A, &B);
                  }
                  __syncthreads();
                  from = ph + 1;
            }
            __syncthreads();
            if (t == 0) s_pos += chunk;
            // bodies appended past this chunk's largest_id are visited next
            p0 = min(p0 + BVT, lid + 1);
      }
      __syncthreads();
      if (t == 0) *count = s_pos - base;
}

// pairs[] = candidates without dropped / merged entries, swapped ones as (p, k)
__global__ void k_pairs_keep(const unsigned char *__restrict__ cflag, int n, int *__restrict__ keep)
{
      int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q < n) keep[q] = (cflag[q] & (F_DROP | F_MERGED)) ? 0 : 1;
}

// Extra (fragment) pairs recorded before candidate position q: the offset of
// the first event at or after q (offsets are cumulative in event order).
__device__ __forceinline__ int x_before(const int *__restrict__ evx, int nev, int nx, int q)
{
      int lo = 0, hi = nev;  // first event with position >= q
      while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (evx[EVX * mid] < q) lo = mid + 1;
            else hi = mid;
      }
      return lo < nev ? evx[EVX * lo + 1] : nx;
}

__global__ void k_pairs_emit(const int *__restrict__ ck, const int *__restrict__ cp,
                             const unsigned char *__restrict__ cflag, const int *__restrict__ pos, int n,
                             const int *__restrict__ evx, int nev, int nx, int *__restrict__ out)
{
      int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q >= n) return;
      unsigned char f = cflag[q];
      if (f & (F_DROP | F_MERGED)) return;
      int o = pos[q] + (nx > 0 ? x_before(evx, nev, nx, q) : 0);
      bool sw = f & F_SWAP;
      out[2 * o] = sw ? cp[q] : ck[q];
      out[2 * o + 1] = sw ? ck[q] : cp[q];
}

// The tail pairs of full fragmentations, spliced in at their events'
// positions: extra pair x of event e goes to pos[q_e] + x.
__global__ void k_pairs_extra(const int *__restrict__ xpairs, int nx, const int *__restrict__ evx, int nev,
                              const int *__restrict__ pos, int *__restrict__ out)
{
      int x = blockIdx.x * blockDim.x + threadIdx.x;
      if (x >= nx) return;
      int lo = 0, hi = nev - 1;  // last event with offset <= x
      while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (evx[EVX * mid + 1] <= x) lo = mid;
            else hi = mid - 1;
      }
      const int o = pos[evx[EVX * lo]] + x;
      out[2 * o] = xpairs[2 * x];
      out[2 * o + 1] = xpairs[2 * x + 1];
}

}  // namespace

DevState dev_state();
int sync_scalars();

static int mesh_alloc(int d)
{
      Ctx &c = ctx();
      if (d < 4 || d % 2 || d > 1200) return NCGPU_E_UNSUPPORTED;  // int cell index up to ~1.7e9
      if (c.crange && c.mesh_d == d) return NCGPU_OK;
      if (c.crange) cudaFree(c.crange);
      size_t dd = (size_t)d;
      c.cell_cap = (dd + 3) * (1 + dd + dd * dd);
      NCG_CK(cudaMalloc(&c.crange, sizeof(int2) * c.cell_cap));
      NCG_CK(cudaMemsetAsync(c.crange, 0xff, sizeof(int2) * c.cell_cap, c.s));
      c.mesh_d = d;
      if (!c.mkeys) {
            size_t N = (size_t)c.n_max;
            NCG_CK(cudaMalloc(&c.mkeys, sizeof(uint32_t) * (N + 1)));
            NCG_CK(cudaMalloc(&c.mvals, sizeof(int) * N));
            NCG_CK(cudaMalloc(&c.mpv, sizeof(int) * N));
            NCG_CK(cudaMalloc(&c.ckey, sizeof(int) * N));
            NCG_CK(cudaMalloc(&c.mcnt, sizeof(int) * (N + 1)));
            NCG_CK(cudaMalloc(&c.moff, sizeof(int) * (N + 2)));
            c.pair_cap = 5L * c.n_max * (long)(c.P.par_how_many_neighbours > 1. ? c.P.par_how_many_neighbours : 16.) + 1024;
            if (c.pair_cap > 0x7fffff00L) c.pair_cap = 0x7fffff00L;
            NCG_CK(cudaMalloc(&c.cand_k, sizeof(int) * c.pair_cap));
            NCG_CK(cudaMalloc(&c.cand_p, sizeof(int) * c.pair_cap));
            NCG_CK(cudaMalloc(&c.cflag, c.pair_cap));
            NCG_CK(cudaMalloc(&c.cpos, sizeof(int) * (c.pair_cap + 1)));
            NCG_CK(cudaMalloc(&c.msums, sizeof(int) * (c.pair_cap / 1024 + 2)));
            c.occ_cap = 64 * c.n_max + 4096;
            NCG_CK(cudaMalloc(&c.occ, sizeof(int) * (size_t)c.occ_cap));
            NCG_CK(cudaMalloc(&c.evx, sizeof(int) * EVX * (size_t)c.ev_cap));
            c.xpair_cap = 4L * c.n_max + 4096;
            NCG_CK(cudaMalloc(&c.xpairs, sizeof(int) * 2 * (size_t)c.xpair_cap));
            NCG_CK(cudaMalloc(&c.xhead, sizeof(int) * N));
            NCG_CK(cudaMemsetAsync(c.xhead, 0xff, sizeof(int) * N, c.s));
            NCG_CK(cudaMalloc(&c.fev, sizeof(int) * (size_t)c.ev_cap));
            NCG_CK(cudaMalloc(&c.vis, sizeof(int) * 3 * (size_t)MAX_VISITS));
            NCG_CK(cudaMalloc(&c.mrec, sizeof(MRec) * N));
            NCG_CK(cudaMalloc(&c.gpart, 4 * sizeof(double) * N));
      }
      return NCGPU_OK;
}

void mesh_free()
{
      Ctx &c = ctx();
      void *ptrs[] = {c.crange, c.mkeys, c.mvals, c.mpv, c.gpart, c.ckey, c.mcnt, c.moff, c.cand_k, c.cand_p, c.cflag, c.cpos,
                      c.occ, c.msums, c.evx, c.xpairs, c.xhead, c.fev, c.vis, c.mrec};
      for (void *p : ptrs)
            if (p) cudaFree(p);
}

__global__ void k_clear_xhead(const int *__restrict__ evx, int nev, int *__restrict__ xhead)
{
      int e = blockIdx.x * blockDim.x + threadIdx.x;
      if (e < nev) xhead[evx[EVX * e + 4]] = -1;
}

int mesh_reset_state()
{
      Ctx &c = ctx();
      if (c.mesh_valid && c.mesh_n > 0) {
            k_cell_clear<<<(c.mesh_n + 255) / 256, 256, 0, c.s>>>(c.mkeys, c.mesh_n, c.crange);
            NCG_LAUNCHED();
      }
      if (c.mesh_nfev > 0) {
            k_clear_xhead<<<(c.mesh_nev + 255) / 256, 256, 0, c.s>>>(c.evx, c.mesh_nev, c.xhead);
            NCG_LAUNCHED();
      }
      c.mesh_valid = 0;
      c.mesh_nev = c.mesh_nfev = c.mesh_nx = c.mesh_nvis = 0;
      return NCGPU_OK;
}

__global__ void k_clear_dirty_events(unsigned char *dirty, const int *ev, int n)
{
      int e = blockIdx.x * blockDim.x + threadIdx.x;
      if (e < n) {
            dirty[ev[3 * e]] = 0;
            dirty[ev[3 * e + 1]] = 0;
      }
}

// The same for the events [0, min(*nev, cap)) counted on the device (grid-stride).
__global__ void k_clear_dirty_events_dev(unsigned char *dirty, const int *ev, const int *nev, int cap)
{
      const int n = min(*nev, cap);
      for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
            dirty[ev[3 * e]] = 0;
            dirty[ev[3 * e + 1]] = 0;
      }
}

// Candidates of the bodies k in [lo, hi) (pop order, positions from base) and
// their hits against the current state: the kernels, without waiting.
static int mesh_segment_launch(const DevState &S, int lid, int lo, int hi, long base, int test)
{
      Ctx &c = ctx();
      cudaStream_t st = c.s;
      const int n = lid + 1;
      const int nb = (n + 255) / 256;
      const int d = c.P.par_collision_cube_cells;
      MRec *rec = (MRec *)c.mrec;
      k_mesh_records<<<nb, 256, 0, st>>>(S, c.mvals, n, rec, c.mpv);
      NCG_LAUNCHED();
      k_mesh_count<<<nb, 256, 0, st>>>(c.mpv, c.ckey, c.mvals, c.crange, lid, lo, hi, d,
                                       (long long)c.cell_cap, c.mcnt);
      NCG_LAUNCHED();
      NCG_TRY(scan_exclusive(c.mcnt, c.moff, n, c.cnt, st));
      if (base > 0) {
            k_add_base<<<(n + 256) / 256, 256, 0, st>>>(c.moff, n, (int)base);
            NCG_LAUNCHED();
      }
      NCG_CK(cudaMemsetAsync(c.scal + S_NHITS, 0, sizeof(int), st));
      // (positions at or past pair_cap are not written: the kernel records the
      // overflow and the host returns NCGPU_E_CAPACITY)
      k_mesh_write<<<(n + MWW * 32 - 1) / (MWW * 32), MWW * 32, 0, st>>>(rec, c.ckey, c.mvals, c.mpv, c.crange, c.moff, lid, lo, hi, d,
                                       (long long)c.cell_cap, c.dt, test, c.cand_k, c.cand_p, c.cflag, c.hi, c.hit_cap,
                                       c.scal + S_NHITS, c.pair_cap, c.err);
      NCG_LAUNCHED();
      return NCGPU_OK;
}

// After mesh_segment_launch and a synchronisation that brought back the
// candidates' end and the hits' count: with hits, the ordered event replay.
// *tot = candidates written.
static int mesh_segment_finish(const DevState &S, int lid, int hi, long base, int end, int nh, const MeshEvArgs &E0,
                               int *tot)
{
      Ctx &c = ctx();
      cudaStream_t st = c.s;
      const long total = (long)end - base;
      if ((long)end > c.pair_cap) return NCGPU_E_CAPACITY;
      *tot = (int)total;
      if (nh > c.hit_cap) return NCGPU_E_CAPACITY;
      if (nh > 0) {
            NCG_CK(cudaMemcpyAsync(c.keys, c.hi, sizeof(int) * (size_t)nh, cudaMemcpyDeviceToDevice, st));
            NCG_CK(cudaMemsetAsync(c.vals, 0, sizeof(int) * (size_t)nh, st));
            NCG_TRY(radix_sort_pairs(c.keys, c.vals, nh, 31, st));
            MeshEvArgs E = E0;
            E.seg_hi = hi;
            MeshFragBufs X{c.evx, c.xpairs, c.xhead, c.fev};
            k_mesh_events<<<1, MEV, 0, st>>>(S, c.cand_k, c.cand_p, c.cflag, c.moff, c.ckey, c.mkeys, c.mvals,
                                             c.crange, (const int *)c.keys, nh, E, c.ev, c.evrec, c.dirty, c.occ,
                                             c.scal + S_NDROP, X, c.err);
            NCG_LAUNCHED();
            k_count_dropped<<<(int)((total + 255) / 256), 256, 0, st>>>(c.cflag + base, (int)total,
                                                                       c.scal + S_NDROP);
            NCG_LAUNCHED();
      }
      return NCGPU_OK;
}

// Both halves with one synchronisation between them.
static int mesh_segment(const DevState &S, int lid, int lo, int hi, long base, int test, const MeshEvArgs &E0,
                        int *tot)
{
      Ctx &c = ctx();
      NCG_TRY(mesh_segment_launch(S, lid, lo, hi, base, test));
      int h2[2] = {0, 0};  // candidates' end, hits
      NCG_CK(cudaMemcpyAsync(&h2[0], c.moff + lid + 1, sizeof(int), cudaMemcpyDeviceToHost, c.s));
      NCG_CK(cudaMemcpyAsync(&h2[1], c.scal + S_NHITS, sizeof(int), cudaMemcpyDeviceToHost, c.s));
      NCG_CK(cudaStreamSynchronize(c.s));
      return mesh_segment_finish(S, lid, hi, base, h2[0], h2[1], E0, tot);
}

// Cell table of the bodies' insertion cells (ckey -> sorted keys, heads).
static int mesh_table(int n)
{
      Ctx &c = ctx();
      cudaStream_t st = c.s;
      NCG_TRY(radix_sort_pairs(c.mkeys, c.mvals, n, 32, st));
      NCG_CK(cudaMemsetAsync(c.mkeys + n, 0xff, sizeof(uint32_t), st));
      k_cell_heads<<<(n + 255) / 256, 256, 0, st>>>(c.mkeys, n, c.crange, c.scal + S_NINS);
      NCG_LAUNCHED();
      return NCGPU_OK;
}

static int read_scal(int idx, int *out)
{
      Ctx &c = ctx();
      NCG_CK(cudaMemcpyAsync(out, c.scal + idx, sizeof(int), cudaMemcpyDeviceToHost, c.s));
      NCG_CK(cudaStreamSynchronize(c.s));
      return NCGPU_OK;
}

// One mesh pass.  test = 1: mesh() (small bodies, predicate and resolution);
// test = 0: get_neighbours_mesh() (every body, no predicate).  With bodies
// larger than the mesh size the pass runs as segments of small bodies (the
// parallel candidate machinery) separated by the big bodies' visits (one CTA
// each); a visit that resolved collisions re-keys the bodies after it, whose
// positions and radii at their turn may have changed.
// defer: for collision types that append no body, leave the pass's counts
// (events, dropped pairs, total_neighbours) to the end of step's read instead
// of reading them back here (mesh_counts_finish).
int mesh_pass(double gam, int test, bool defer)
{
      Ctx &c = ctx();
      cudaStream_t st = c.s;
      const int d = c.P.par_collision_cube_cells;
      NCG_TRY(mesh_alloc(d));
      NCG_TRY(mesh_reset_state());
      const int lid = c.largest_id;
      const int n = lid + 1;
      // counters of the pass cleared on the device (no host copy on the step's path)
      NCG_CK(cudaMemsetAsync(c.scal + S_NHITS, 0, 2 * sizeof(int), st));    // NHITS, NEV
      NCG_CK(cudaMemsetAsync(c.scal + S_NBIG, 0, 3 * sizeof(int), st));     // NBIG, NDROP, NINS
      NCG_CK(cudaMemsetAsync(c.scal + S_NXPAIRS, 0, 3 * sizeof(int), st));  // NXPAIRS, NSKIP, NFEV
      c.n_cand = c.n_pairs = 0;
      c.total_neighbours = 0;
      c.how_many_small = c.how_many_big = 0;
      c.mesh_nvis = 0;
      if (n <= 0) return sync_scalars();
      DevState S = dev_state();
      const double half = gam * (double)d / 2.0;
      const int nb = (n + 255) / 256;
      k_mesh_keys<<<nb, 256, 0, st>>>(S, lid, gam, half, d, !test, c.mkeys, c.mvals, c.ckey, c.scal + S_NBIG);
      NCG_LAUNCHED();
      NCG_TRY(mesh_table(n));
      c.mesh_valid = 1;
      c.mesh_n = n;
      // the pass as one segment of every body, its candidates launched before
      // the count of bodies larger than the mesh size comes back (with the
      // candidates' end and the hits, one synchronisation); with such bodies
      // the segmented pass below starts over
      NCG_TRY(mesh_segment_launch(S, lid, 0, lid + 1, 0, test));
      int h3[3] = {0, 0, 0};  // bodies larger than the mesh size, candidates' end, hits
      NCG_CK(cudaMemcpyAsync(&h3[0], c.scal + S_NBIG, sizeof(int), cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaMemcpyAsync(&h3[1], c.moff + n, sizeof(int), cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaMemcpyAsync(&h3[2], c.scal + S_NHITS, sizeof(int), cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaStreamSynchronize(st));
      const int nbig = h3[0];
      MeshEvArgs E{lid, d, c.P.par_collision_type, c.P.par_one_collision_only_bool, c.P.par_mesh_bool, c.ev_cap,
                   c.n_max, c.occ_cap, n, (long long)c.cell_cap, c.dt, c.P.par_collision_parameter,
                   c.P.par_mutual_bool, c.xpair_cap, FragArgs{}, lid + 1};
      if (test && E.type == NCGPU_COLLISION_FRAGMENTATION && !make_frag_args(c, E.frag)) return NCGPU_E_ARG;
      long base = 0, small_total = 0;
      int ev_clean = 0;  // events whose dirty marks are cleared
      auto clear_dirty = [&](int nev) -> int {
            const int hi = min(nev, c.ev_cap);
            if (hi > ev_clean) {
                  k_clear_dirty_events<<<(hi - ev_clean + 255) / 256, 256, 0, st>>>(c.dirty, c.ev + 3 * (size_t)ev_clean,
                                                                                  hi - ev_clean);
                  NCG_LAUNCHED();
                  ev_clean = hi;
            }
            return NCGPU_OK;
      };
      if (!test || nbig == 0) {
            int tot = 0;
            NCG_TRY(mesh_segment_finish(S, lid, lid + 1, 0, h3[1], h3[2], E, &tot));
            base = small_total = tot;
      } else {
            int s = 0;
            bool rekey = false;
            for (;;) {
                  int e = 0x7fffffff;
                  NCG_CK(cudaMemcpyAsync(c.n_dev, &e, sizeof(int), cudaMemcpyHostToDevice, st));
                  k_next_big<<<(lid - s + 256) / 256, 256, 0, st>>>(S, s, lid, gam, c.n_dev);
                  NCG_LAUNCHED();
                  NCG_CK(cudaMemcpyAsync(&e, c.n_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
                  NCG_CK(cudaStreamSynchronize(st));
                  const int hi = e == 0x7fffffff ? lid + 1 : e;
                  if (hi > s) {
                        if (rekey) {
                              k_cell_clear<<<nb, 256, 0, st>>>(c.mkeys, n, c.crange);
                              NCG_LAUNCHED();
                              k_mesh_rekey<<<nb, 256, 0, st>>>(S, s, lid, gam, half, d, c.mkeys, c.mvals, c.ckey);
                              NCG_LAUNCHED();
                              NCG_TRY(mesh_table(n));
                              rekey = false;
                        }
                        int tot = 0;
                        NCG_TRY(mesh_segment(S, lid, s, hi, base, test, E, &tot));
                        base += tot;
                        small_total += tot;
                        int nev = 0;
                        NCG_TRY(read_scal(S_NEV, &nev));
                        NCG_TRY(clear_dirty(nev));
                  }
                  if (e == 0x7fffffff) break;
                  int nev0 = 0, nev1 = 0, cnt = 0;
                  NCG_TRY(read_scal(S_NEV, &nev0));
                  MeshFragBufs X{c.evx, c.xpairs, c.xhead, c.fev};
                  k_big_visit<<<1, BVT, 0, st>>>(S, e, gam, (int)base, c.pair_cap, E, c.cand_k, c.cand_p, c.cflag,
                                                 c.ev, c.evrec, X, c.n_dev, c.err);
                  NCG_LAUNCHED();
                  NCG_CK(cudaMemcpyAsync(&cnt, c.n_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
                  NCG_TRY(read_scal(S_NEV, &nev1));
                  if (c.mesh_nvis < MAX_VISITS) {
                        c.vis_host[3 * c.mesh_nvis] = e;
                        c.vis_host[3 * c.mesh_nvis + 1] = (int)base;
                        c.vis_host[3 * c.mesh_nvis + 2] = (int)base + cnt;
                  }
                  c.mesh_nvis++;
                  base += cnt;
                  if (base > c.pair_cap) return NCGPU_E_CAPACITY;
                  rekey = rekey || nev1 > nev0;
                  s = e + 1;
                  if (s > lid) break;
            }
            if (c.mesh_nvis > MAX_VISITS) return NCGPU_E_CAPACITY;
            if (c.mesh_nvis > 0)
                  NCG_CK(cudaMemcpyAsync(c.vis, c.vis_host, sizeof(int) * 3 * (size_t)c.mesh_nvis,
                                         cudaMemcpyHostToDevice, st));
      }
      if (defer && test && nbig == 0 && E.type != NCGPU_COLLISION_FRAGMENTATION) {
            k_clear_dirty_events_dev<<<32, 256, 0, st>>>(c.dirty, c.ev, c.scal + S_NEV, c.ev_cap);
            NCG_LAUNCHED();
            c.n_cand = (int)base;
            c.mesh_nfev = 0;  // (no fragments without the fragmentation model)
            c.mesh_nx = 0;
            c.how_many_big = 0;
            c.mesh_pending = 1;
            c.mesh_base = base;
            c.mesh_small_total = small_total;
            return NCGPU_OK;
      }
      int h[S_COUNT];
      NCG_TRY(sync_scalars_h(h));
      NCG_TRY(clear_dirty(c.n_events));
      c.n_cand = (int)base;
      c.mesh_nev = min(c.n_events, c.ev_cap);
      c.mesh_nfev = h[S_NFEV];
      c.mesh_nx = h[S_NXPAIRS];
      c.total_neighbours = small_total - h[S_NDROP];
      c.n_pairs = c.P.par_mutual_bool ? (int)(base - h[S_NDROP] - h[S_NSKIP] + h[S_NXPAIRS]) : 0;
      c.how_many_big = test ? c.mesh_nvis : 0;
      return NCGPU_OK;
}

// The counts of a deferred mesh pass from the device scalars h (S_COUNT ints).
void mesh_counts_finish(const int *h)
{
      Ctx &c = ctx();
      if (!c.mesh_pending) return;
      c.mesh_pending = 0;
      c.n_events = h[S_NEV];
      c.collision_count = h[S_CCOUNT];
      c.mesh_nev = min(c.n_events, c.ev_cap);
      c.total_neighbours = c.mesh_small_total - h[S_NDROP];
      c.n_pairs = c.P.par_mutual_bool ? (int)(c.mesh_base - h[S_NDROP] - h[S_NSKIP] + h[S_NXPAIRS]) : 0;
}

}  // namespace ncg

using namespace ncg;

extern "C" int ncgpu_mesh(double gam, int with_collisions, int *n_pairs, int *n_events, long *total_neighbours)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      if (!(gam > 0.)) return NCGPU_E_ARG;
      NCG_TRY(mesh_pass(gam, with_collisions ? 1 : 0, false));
      if (n_pairs) *n_pairs = c.n_pairs;
      if (n_events) *n_events = with_collisions ? c.n_events : 0;
      if (total_neighbours) *total_neighbours = c.total_neighbours;
      return NCGPU_OK;
}

extern "C" int ncgpu_get_pairs(struct ncgpu_pair *out, int cap, int *n)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited) return NCGPU_E_STATE;
      if (!n) return NCGPU_E_ARG;
      *n = c.n_pairs;
      if (!out || cap <= 0 || c.n_cand == 0 || c.n_pairs == 0) return NCGPU_OK;
      cudaStream_t st = c.s;
      const int nc = c.n_cand;
      const int nb = (nc + 255) / 256;
      k_pairs_keep<<<nb, 256, 0, st>>>(c.cflag, nc, c.cpos);
      NCG_LAUNCHED();
      NCG_TRY(scan_exclusive(c.cpos, c.cpos, nc, c.msums, st));  // in place
      int *dst = nullptr;
      NCG_CK(cudaMalloc(&dst, sizeof(int) * 2 * (size_t)c.n_pairs));
      k_pairs_emit<<<nb, 256, 0, st>>>(c.cand_k, c.cand_p, c.cflag, c.cpos, nc, c.evx, c.mesh_nev, c.mesh_nx, dst);
      NCG_LAUNCHED();
      if (c.mesh_nx > 0) {
            k_pairs_extra<<<(c.mesh_nx + 255) / 256, 256, 0, st>>>(c.xpairs, c.mesh_nx, c.evx, c.mesh_nev, c.cpos, dst);
            NCG_LAUNCHED();
      }
      const int k = c.n_pairs < cap ? c.n_pairs : cap;
      cudaError_t e = cudaMemcpyAsync(out, dst, sizeof(int) * 2 * (size_t)k, cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      cudaFree(dst);
      if (e != cudaSuccess) return cuda_fail(e, "ncgpu_get_pairs copy", __FILE__, __LINE__);
      return NCGPU_OK;
}

extern "C" int ncgpu_mesh_reset(void)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited) return NCGPU_E_STATE;
      return mesh_reset_state();
}
