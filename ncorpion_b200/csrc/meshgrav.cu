// Mesh-mode pieces of the step: the three largest bodies moved to slots 0-2
// and the mesh gravity field.
//
// three_largest_moonlets (src/structure.c:914-1002) scans slots in order; the
// first three existing bodies are ranked by special rules, every later body
// displaces a ranked one only when strictly larger, so the result is the
// first three of a stable sort (radius descending) of [ranked three, later
// bodies in slot order].  The later bodies' top three by (radius desc, slot
// asc) come from a parallel reduction; one thread merges and then applies
// three_largest_three_first (src/structure.c:1005-1063).
//
// Mesh gravity (vector_field's mesh branches, src/physics.c:84-109, 205-261,
// 297-379): central mass, the three largest bodies against every body, and
// pairs[].  A body's pairs[] contributions are, in list order, its own pops
// (cells 26..0, lower indices ascending) followed by the later bodies whose
// pops found it, in ascending index.  Each thread walks the cells of its own
// body in exactly that order, so the FP64 sums match the reference without
// reading pairs[]; the three bodies 0-2 and CM_acc sum every body's term in
// slot order (sequential chains in the exact mode).
#include <algorithm>
#include "common.cuh"
#include "physics.cuh"

namespace ncg {

DevState dev_state();
int sync_scalars();

namespace {

struct Top3 {
      double R[3];
      int i[3];
};

__device__ __forceinline__ bool better(double Ra, int ia, double Rb, int ib)
{
      return Ra > Rb || (Ra == Rb && ia < ib);
}

__device__ __forceinline__ void t3_insert(Top3 &t, double R, int i)
{
      if (i < 0) return;
      if (t.i[0] < 0 || better(R, i, t.R[0], t.i[0])) {
            t.R[2] = t.R[1]; t.i[2] = t.i[1]; t.R[1] = t.R[0]; t.i[1] = t.i[0]; t.R[0] = R; t.i[0] = i;
      } else if (t.i[1] < 0 || better(R, i, t.R[1], t.i[1])) {
            t.R[2] = t.R[1]; t.i[2] = t.i[1]; t.R[1] = R; t.i[1] = i;
      } else if (t.i[2] < 0 || better(R, i, t.R[2], t.i[2])) {
            t.R[2] = R; t.i[2] = i;
      }
}

// first three existing slots (one warp, ballots over 32 slots at a time)
__global__ void k_first3(const int *__restrict__ ex, int lid, int *__restrict__ out)
{
      int lane = threadIdx.x, found = 0;
      int e[3] = {-1, -1, -1};
      for (int base = 0; base <= lid && found < 3; base += 32) {
            int j = base + lane;
            unsigned m = __ballot_sync(0xffffffffu, j <= lid && ex[j]);
            while (m && found < 3) {
                  int b = __ffs(m) - 1;
                  e[found++] = base + b;
                  m &= m - 1;
            }
      }
      if (lane == 0) {
            out[0] = e[0];
            out[1] = e[1];
            out[2] = e[2];
      }
}

constexpr int TB = 256;

// top three by (radius desc, slot asc) of existing slots > first3[2]
__global__ void k_top3_part(const DevState S, int lid, const int *__restrict__ first3, double *__restrict__ partR,
                            int *__restrict__ parti)
{
      __shared__ double sR[3][TB];
      __shared__ int si[3][TB];
      Top3 t;
      for (int q = 0; q < 3; q++) { t.R[q] = 0.; t.i[q] = -1; }
      const int start = first3[2] + 1;
      if (first3[2] >= 0) {
            // four slots a round, their loads issued together (the top three of a
            // total order do not depend on the order of the insertions)
            const int stride = gridDim.x * TB;
            int j = start + blockIdx.x * TB + threadIdx.x;
            for (; j + 3 * stride <= lid; j += 4 * stride) {
                  int e[4];
                  double r[4];
#pragma unroll
                  for (int u = 0; u < 4; u++) {
                        e[u] = S.ex[j + u * stride];
                        r[u] = S.R[j + u * stride];
                  }
#pragma unroll
                  for (int u = 0; u < 4; u++)
                        if (e[u]) t3_insert(t, r[u], j + u * stride);
            }
            for (; j <= lid; j += stride)
                  if (S.ex[j]) t3_insert(t, S.R[j], j);
      }
      for (int q = 0; q < 3; q++) { sR[q][threadIdx.x] = t.R[q]; si[q][threadIdx.x] = t.i[q]; }
      __syncthreads();
      for (int o = TB / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) {
                  Top3 u;
                  for (int q = 0; q < 3; q++) { u.R[q] = sR[q][threadIdx.x]; u.i[q] = si[q][threadIdx.x]; }
                  for (int q = 0; q < 3; q++) t3_insert(u, sR[q][threadIdx.x + o], si[q][threadIdx.x + o]);
                  for (int q = 0; q < 3; q++) { sR[q][threadIdx.x] = u.R[q]; si[q][threadIdx.x] = u.i[q]; }
            }
            __syncthreads();
      }
      if (threadIdx.x < 3) {
            partR[blockIdx.x * 3 + threadIdx.x] = sR[threadIdx.x][0];
            parti[blockIdx.x * 3 + threadIdx.x] = si[threadIdx.x][0];
      }
}

__device__ void swap_bodies(const DevState &S, int a, int b)
{
      double *f[8] = {S.x, S.y, S.z, S.vx, S.vy, S.vz, S.m, S.R};
      for (int q = 0; q < 8; q++) {
            double t = f[q][a];
            f[q][a] = f[q][b];
            f[q][b] = t;
      }
}

__device__ void move_body(const DevState &S, int dst, int src)
{
      double *f[8] = {S.x, S.y, S.z, S.vx, S.vy, S.vz, S.m, S.R};
      for (int q = 0; q < 8; q++) f[q][dst] = f[q][src];
}

// merge + three_largest_three_first; out[0..2] = three_largest_indexes
__global__ void k_top3_final(const DevState S, const int *__restrict__ first3, const double *__restrict__ partR,
                             const int *__restrict__ parti, int nparts, int mesh_bool, int *__restrict__ out)
{
      // later bodies' top three: the block partials folded by the warp (the order
      // (radius desc, slot asc) is total, so any folding order gives the same three)
      Top3 rest;
      for (int q = 0; q < 3; q++) { rest.R[q] = 0.; rest.i[q] = -1; }
      for (int b = threadIdx.x; b < nparts; b += 32)
            for (int q = 0; q < 3; q++) t3_insert(rest, partR[3 * b + q], parti[3 * b + q]);
      for (int o = 16; o > 0; o >>= 1) {
            double oR[3];
            int oi[3];
            for (int q = 0; q < 3; q++) {
                  oR[q] = __shfl_down_sync(0xffffffffu, rest.R[q], o);
                  oi[q] = __shfl_down_sync(0xffffffffu, rest.i[q], o);
            }
            for (int q = 0; q < 3; q++) t3_insert(rest, oR[q], oi[q]);
      }
      if (threadIdx.x != 0) return;
      int e0 = first3[0], e1 = first3[1], e2 = first3[2];
      int t[3] = {-1, -1, -1};
      double R0 = 0., R1 = 0., R2 = 0., R;
      // the first three existing bodies (src/structure.c:933-978)
      if (e0 >= 0) { R0 = S.R[e0]; t[0] = e0; }
      if (e1 >= 0) {
            R1 = S.R[e1];
            if (R0 > R1) t[1] = e1;
            else { t[1] = t[0]; t[0] = e1; R = R1; R1 = R0; R0 = R; }
      }
      if (e2 >= 0) {
            R2 = S.R[e2];
            if (R1 >= R2) t[2] = e2;
            else if (R2 > R1 && R2 <= R0) { t[2] = t[1]; t[1] = e2; R = R2; R2 = R1; R1 = R; }
            else { t[2] = t[1]; t[1] = t[0]; t[0] = e2; R = R2; R2 = R1; R1 = R0; R0 = R; }
      }
      // later bodies, strictly-larger insertion in (radius desc, slot asc) order
      for (int q = 0; q < 3; q++) {
            int j = rest.i[q];
            if (j < 0 || e2 < 0) continue;
            double Rj = rest.R[q];
            if (Rj > R0) { t[2] = t[1]; t[1] = t[0]; t[0] = j; R2 = R1; R1 = R0; R0 = Rj; }
            else if (Rj > R1) { t[2] = t[1]; t[1] = j; R2 = R1; R1 = Rj; }
            else if (Rj > R2) { t[2] = j; R2 = Rj; }
      }
      out[0] = t[0]; out[1] = t[1]; out[2] = t[2];
      if (t[0] < 0 || t[1] < 0 || t[2] < 0) return;  // fewer than three bodies
      // three_largest_three_first
      int first = t[0], second = t[1], third = t[2];
      if (first != 0) {
            if (S.ex[0]) swap_bodies(S, 0, first);
            else { move_body(S, 0, first); d_lose(S, first, mesh_bool); S.ex[0] = 1; }
            if (second == 0) second = first;
            else if (third == 0) third = first;
      }
      if (second != 1) {
            if (S.ex[1]) swap_bodies(S, 1, second);
            else { move_body(S, 1, second); d_lose(S, second, mesh_bool); S.ex[1] = 1; }
            if (third == 1) third = second;
      }
      if (third != 2) {
            if (S.ex[2]) swap_bodies(S, 2, third);
            else { move_body(S, 2, third); d_lose(S, third, mesh_bool); S.ex[2] = 1; }
      }
}

}  // namespace

namespace {

__device__ __forceinline__ long long g_noff(int l, int d)
{
      int di = l % 3 - 1, dj = (l / 3) % 3 - 1, dk = l / 9 - 1;
      return di + dj * (long long)d + dk * (long long)d * d;
}

// a + ((G*m_o) * (x_o - x_b)) / D^3 with the reference's operation order
__device__ __forceinline__ void pair_add(const DevState &S, int b, int o, double G, double sp, bool soft, double &ax,
                                         double &ay, double &az)
{
      double dx = DSUB(S.x[o], S.x[b]), dy = DSUB(S.y[o], S.y[b]), dz = DSUB(S.z[o], S.z[b]);
      double r2 = DADD(DADD(DMUL(dx, dx), DMUL(dy, dy)), DMUL(dz, dz));
      if (soft) {
            double s = DMUL(sp, DADD(S.R[b], S.R[o]));
            r2 = DADD(r2, DMUL(s, s));
      }
      double D = __dsqrt_rn(r2);
      double D3 = DMUL(DMUL(D, D), D);
      double g = DMUL(G, S.m[o]);
      const double y = __drcp_rn(D3);  // the three quotients by D3 share RN(1/D3)
      ax = DADD(ax, div_by_recip(DMUL(g, dx), D3, y));
      ay = DADD(ay, div_by_recip(DMUL(g, dy), D3, y));
      az = DADD(az, div_by_recip(DMUL(g, dz), D3, y));
}

// A body's gravity fields in a cell-ordered copy (64 bytes), read by the walk
// instead of gathering each field from the state arrays.
struct __align__(16) GRec {
      double x, y, z, mp;  // mp: the mass of a pairs[] partner (existing, not one of bodies 0..2), else 0
      double m, R, pad0;
      int ex, partner;
};

// gp (when not null): the partners' x, y, z and partner mass alone, 32 bytes a
// position, which the fast walk reads for every pair term.
__global__ void k_grav_records(const DevState S, const int *__restrict__ vals, int n, GRec *__restrict__ rec,
                               double4 *__restrict__ gp)
{
      int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q >= n) return;
      const int b = vals[q];
      GRec r;
      r.x = S.x[b]; r.y = S.y[b]; r.z = S.z[b]; r.m = S.m[b]; r.R = S.R[b];
      r.pad0 = 0.;
      r.ex = S.ex[b];
      r.partner = (b > 2 && r.ex) ? 1 : 0;
      r.mp = r.partner ? r.m : 0.;
      rec[q] = r;
      if (gp) gp[q] = make_double4(r.x, r.y, r.z, r.mp);
}

// pair_add with the partner's fields from its record (same operations)
__device__ __forceinline__ void pair_add_rec(double xb, double yb, double zb, double Rb, const GRec &o, double G,
                                             double sp, bool soft, double &ax, double &ay, double &az)
{
      double dx = DSUB(o.x, xb), dy = DSUB(o.y, yb), dz = DSUB(o.z, zb);
      double r2 = DADD(DADD(DMUL(dx, dx), DMUL(dy, dy)), DMUL(dz, dz));
      if (soft) {
            double s = DMUL(sp, DADD(Rb, o.R));
            r2 = DADD(r2, DMUL(s, s));
      }
      double D = __dsqrt_rn(r2);
      double D3 = DMUL(DMUL(D, D), D);
      double g = DMUL(G, o.m);
      const double y = __drcp_rn(D3);
      ax = DADD(ax, div_by_recip(DMUL(g, dx), D3, y));
      ay = DADD(ay, div_by_recip(DMUL(g, dy), D3, y));
      az = DADD(az, div_by_recip(DMUL(g, dz), D3, y));
}

struct MGArgs {
      int lid, d, central, mutual, soft;
      long long cell_cap;
      double G, sp;
      const double *cm;         // the central mass's record (device): x, y, z at 0..2, mass at 6
      int lid0;                 // largest_id of the mesh pass (slots in the cell table)
      int nt;                   // N_tilde
      int nfev;                 // full fragmentations of the pass
      const int *evx, *fev, *xhead;
      int nvis;                 // visits of bodies larger than the mesh size
      const int *vis;           // (body, first, end) candidate positions, in visit order
      const int *cp;            // candidate partners (a visit's list ascends)
      J2Arg j2;                 // the central body's J2 term
      int cellterms;            // terms of bodies 0..2 and CM_acc at the walk's (cell-order)
                                // position, for the parallel sums; else at the slot (exact chains)
};

// CM_acc's chain c (0..2) in `terms`: after the 9 chains of bodies 0..2, one
// term per slot, or two (central, J2) with J2, in the reference's order.
__device__ __forceinline__ double *cm_chain(double *terms, const MGArgs &A, long N, int c)
{
      return terms + 9 * N + (size_t)c * (A.j2.on ? 2 : 1) * N;
}

// Whether b is in the candidate list cp[lo, hi) (ascending).
__device__ __forceinline__ bool in_list(const int *__restrict__ cp, int lo, int hi, int b)
{
      while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const int v = cp[mid];
            if (v < b) lo = mid + 1;
            else if (v > b) hi = mid;
            else return true;
      }
      return false;
}

// The tail fragments of full fragmentation e (EVX record): slots
// fid0 .. fid0 + nt - 1.  Adds, in pairs[] order, the terms of the largest
// fragment A and of the tail (except `self`) to body b.
__device__ __forceinline__ void tail_terms(const DevState &S, const MGArgs &A, int e, int self, int b,
                                           double &ax, double &ay, double &az)
{
      const int *r = A.evx + (size_t)EVX * e;
      const int fid0 = r[3], big = r[4];
      if (big != self && big > 2 && S.ex[big]) pair_add(S, b, big, A.G, A.sp, A.soft, ax, ay, az);
      for (int n = 0; n < A.nt; n++) {
            const int f = fid0 + n;
            if (f != self && f > 2 && S.ex[f]) pair_add(S, b, f, A.G, A.sp, A.soft, ax, ay, az);
      }
}

// A body's terms that do not come from pairs[]: the central mass (its
// acceleration and, with J2, the J2 share; CM_acc's terms) and the three
// largest bodies 0..2 (b's acceleration from them, their terms from b), with
// the reference's operations.  Writes the per-body terms at ti; returns false
// when the body has nothing more to add (empty slot, or one of bodies 0..2).
// tv (when not null): the body's terms of the 12 chains (bodies 0..2's
// components, then CM_acc's, the J2 term added to the central one) returned
// instead of stored in terms; zero where the body adds none.
__device__ __forceinline__ bool body_prologue(const DevState &S, const MGArgs &A, const GRec &me, int b, long ti,
                                              double *__restrict__ terms, long N, double *__restrict__ ax,
                                              double *__restrict__ ay, double *__restrict__ az, double &a_x,
                                              double &a_y, double &a_z, double *tv = nullptr)
{
      const int f = A.j2.on ? 2 : 1;
      a_x = a_y = a_z = 0.;
      if (tv)
            for (int w = 0; w < 12; w++) tv[w] = 0.;
      if (!me.ex) {
            if (tv) return false;
            // an empty slot adds +0.0 to every chain (they then read all terms
            // without looking at exists[])
            for (int w = 0; w < 9; w++) terms[(size_t)w * N + ti] = 0.;
            for (int c = 0; c < 3; c++)
                  for (int u = 0; u < f; u++) cm_chain(terms, A, N, c)[f * ti + u] = 0.;
            return false;
      }
      if (A.central) {
            const double mu = DMUL(A.G, A.cm[6]);
            double DX = DSUB(me.x, A.cm[0]), DY = DSUB(me.y, A.cm[1]), DZ = DSUB(me.z, A.cm[2]);
            double rk = __dsqrt_rn(DADD(DADD(DMUL(DX, DX), DMUL(DY, DY)), DMUL(DZ, DZ)));
            double r3 = DMUL(DMUL(rk, rk), rk);
            const double y3 = __drcp_rn(r3);  // the six quotients by r3 share RN(1/r3)
            a_x = div_by_recip(DMUL(-mu, DX), r3, y3);
            a_y = div_by_recip(DMUL(-mu, DY), r3, y3);
            a_z = div_by_recip(DMUL(-mu, DZ), r3, y3);
            double g = DMUL(A.G, me.m);
            const double cc[3] = {div_by_recip(DMUL(g, DX), r3, y3), div_by_recip(DMUL(g, DY), r3, y3),
                                  div_by_recip(DMUL(g, DZ), r3, y3)};
            double cj[3] = {0., 0., 0.};
            if (A.j2.on) d_j2(A.j2, mu, DX, DY, DZ, rk, r3, me.m, a_x, a_y, a_z, cj);  // src/physics.c:149-160
            for (int c = 0; c < 3; c++) {
                  if (tv) {
                        tv[9 + c] = A.j2.on ? cc[c] + cj[c] : cc[c];
                  } else {
                        cm_chain(terms, A, N, c)[f * ti] = cc[c];
                        if (A.j2.on) cm_chain(terms, A, N, c)[2 * ti + 1] = cj[c];
                  }
            }
      }
      if (b <= 2) {  // bodies 0..2: central term only here
            ax[b] = a_x; ay[b] = a_y; az[b] = a_z;
            if (A.cellterms && !tv)  // (the parallel sums read every position)
                  for (int w = 0; w < 9; w++) terms[(size_t)w * N + ti] = 0.;
            return false;
      }
      if (A.mutual) {
            const double xb = me.x, yb = me.y, zb = me.z, Rb = me.R, mb = me.m;
            for (int i = 0; i < 3; i++) {
                  if (!S.ex[i]) continue;
                  // body b's term from i and i's term from b (G*m_b*(X_b - X_i)/D^3,
                  // src/physics.c:216-257) share D^3: the squared differences and
                  // the softening are the same numbers
                  double dx = DSUB(S.x[i], xb), dy = DSUB(S.y[i], yb), dz = DSUB(S.z[i], zb);
                  double r2 = DADD(DADD(DMUL(dx, dx), DMUL(dy, dy)), DMUL(dz, dz));
                  if (A.soft) {
                        double sft = DMUL(A.sp, DADD(Rb, S.R[i]));
                        r2 = DADD(r2, DMUL(sft, sft));
                  }
                  const double D = __dsqrt_rn(r2);
                  const double D3 = DMUL(DMUL(D, D), D);
                  const double gi = DMUL(A.G, S.m[i]), gb = DMUL(A.G, mb);
                  const double y = __drcp_rn(D3);
                  a_x = DADD(a_x, div_by_recip(DMUL(gi, dx), D3, y));
                  a_y = DADD(a_y, div_by_recip(DMUL(gi, dy), D3, y));
                  a_z = DADD(a_z, div_by_recip(DMUL(gi, dz), D3, y));
                  const double t3[3] = {div_by_recip(DMUL(gb, DSUB(xb, S.x[i])), D3, y),
                                        div_by_recip(DMUL(gb, DSUB(yb, S.y[i])), D3, y),
                                        div_by_recip(DMUL(gb, DSUB(zb, S.z[i])), D3, y)};
                  for (int c = 0; c < 3; c++) {
                        if (tv) tv[3 * i + c] = t3[c];
                        else terms[(3 * i + c) * N + ti] = t3[c];
                  }
            }
      }
      return true;
}

// Accelerations of bodies 3..lid (bodies 0..2 are finished by k_mesh_big3);
// terms for bodies 0..2 and CM_acc go to `terms` (12 blocks of n_max, the
// CM_acc ones doubled with J2).  Every body's pair terms are added in pairs[]
// order (the exact mode's kernel).
__global__ void k_mesh_grav(DevState S, MGArgs A, const int *__restrict__ ckey, const uint32_t *__restrict__ keys,
                            const int *__restrict__ vals, const int2 *__restrict__ crange, int have_cells,
                            const GRec *__restrict__ grec, double *__restrict__ ax, double *__restrict__ ay,
                            double *__restrict__ az, double *__restrict__ terms, long N)
{
      // bodies of the cell table in cell order (neighbouring threads share cells
      // and partners), then the bodies appended after the pass
      const int t = blockIdx.x * blockDim.x + threadIdx.x;
      if (t > A.lid) return;
      const bool incell = have_cells && t <= A.lid0;
      const int b = incell ? vals[t] : t;
      const long ti = A.cellterms ? t : b;  // where this body's terms go (coalesced in cell order)
      // this body's fields, loaded once: from its cell-ordered record (one
      // contiguous 64-byte read; the same values as the state arrays)
      GRec me;
      if (incell) {
            me = grec[t];
      } else {
            me.x = S.x[b]; me.y = S.y[b]; me.z = S.z[b]; me.m = S.m[b]; me.R = S.R[b];
            me.ex = S.ex[b];
      }
      double a_x, a_y, a_z;
      if (!body_prologue(S, A, me, b, ti, terms, N, ax, ay, az, a_x, a_y, a_z)) return;
      if (A.mutual && have_cells && b > A.lid0) {
            // a tail fragment created by the pass: its pairs are those of its
            // fragmentation (the largest fragment, then the other tail bodies)
            int lo = 0, hi = A.nfev - 1;  // last full fragmentation with fid0 <= b
            while (lo < hi) {
                  int mid = (lo + hi + 1) >> 1;
                  if (A.evx[(size_t)EVX * A.fev[mid] + 3] <= b) lo = mid;
                  else hi = mid - 1;
            }
            if (A.nfev > 0) {
                  const int e = A.fev[lo];
                  const int fid0 = A.evx[(size_t)EVX * e + 3];
                  if (b >= fid0 && b < fid0 + A.nt) tail_terms(S, A, e, b, b, a_x, a_y, a_z);
            }
      }
      const int L = (have_cells && b <= A.lid0) ? ckey[b] : -1;
      if (A.mutual && have_cells) {
            // full fragmentations whose largest fragment is b: their tail pairs
            // follow the event's own candidate (k, p) in b's sequence
            int xe = A.xhead ? A.xhead[b] : -1;
            auto anchor = [&](int k, int p) {
                  while (xe >= 0 && A.evx[(size_t)EVX * xe + 6] == k && A.evx[(size_t)EVX * xe + 7] == p) {
                        tail_terms(S, A, xe, b, b, a_x, a_y, a_z);
                        xe = A.evx[(size_t)EVX * xe + 5];
                  }
            };
            // a big body's visit that listed b (pairs[] holds (e, b) at e's turn)
            auto visit_term = [&](int v) {
                  const int e = A.vis[3 * v];
                  if (!in_list(A.cp, A.vis[3 * v + 1], A.vis[3 * v + 2], b)) return;
                  if (e > 2 && S.ex[e]) pair_add(S, b, e, A.G, A.sp, A.soft, a_x, a_y, a_z);
                  anchor(e, b);
            };
            // visits of big bodies before b
            int vi = 0;
            for (; vi < A.nvis && A.vis[3 * vi] < b; ++vi) visit_term(vi);
            // b's own visit (b larger than the mesh size) replaces its pops
            if (vi < A.nvis && A.vis[3 * vi] == b) {
                  for (int r = A.vis[3 * vi + 1]; r < A.vis[3 * vi + 2]; ++r) {
                        const int p = A.cp[r];
                        if (p > 2 && S.ex[p]) pair_add(S, b, p, A.G, A.sp, A.soft, a_x, a_y, a_z);
                        anchor(b, p);
                  }
                  ++vi;
            }
            if (L >= 0) {
                  const double xb = me.x, yb = me.y, zb = me.z, Rb = me.R;
                  // own pops: cells 26..0, lower indices ascending
                  int cur[27];
                  for (int l = 26; l >= 0; --l) {
                        long long cell = L + g_noff(l, A.d);
                        cur[l] = -1;
                        if (cell < 0 || cell >= A.cell_cap) continue;
                        int s = crange[cell].x;
                        if (s < 0) continue;
                        int q = s;
                        for (; keys[q] == (uint32_t)cell; ++q) {
                              int p = vals[q];
                              if (p >= b) break;
                              if (p > 2 && grec[q].ex) pair_add_rec(xb, yb, zb, Rb, grec[q], A.G, A.sp, A.soft, a_x, a_y, a_z);
                              anchor(b, p);
                        }
                        cur[l] = (keys[q] == (uint32_t)cell) ? q : -1;  // first higher index, if any
                  }
                  // later bodies that found b, ascending index: 27-way merge, with
                  // the later big bodies' visits in index order
                  for (;;) {
                        int best = 0x7fffffff, bl = -1;
                        for (int l = 0; l < 27; ++l) {
                              int q = cur[l];
                              if (q < 0) continue;
                              int v = vals[q];
                              if (v < best) { best = v; bl = l; }
                        }
                        for (; vi < A.nvis && A.vis[3 * vi] < best; ++vi) visit_term(vi);
                        if (bl < 0) break;
                        const int qb = cur[bl];
                        if (best > 2 && best != b && grec[qb].ex)
                              pair_add_rec(xb, yb, zb, Rb, grec[qb], A.G, A.sp, A.soft, a_x, a_y, a_z);
                        anchor(best, b);
                        long long cell = L + g_noff(bl, A.d);
                        int q = cur[bl] + 1;
                        cur[bl] = (keys[q] == (uint32_t)cell) ? q : -1;
                  }
            }
            for (; vi < A.nvis; ++vi) visit_term(vi);
            for (; xe >= 0; xe = A.evx[(size_t)EVX * xe + 5]) tail_terms(S, A, xe, b, b, a_x, a_y, a_z);
      }
      ax[b] = a_x; ay[b] = a_y; az[b] = a_z;
}

// The fast modes' mesh gravity, for passes without bodies larger than the
// mesh size and without fragments appended: a body's pairs[] partners are then
// exactly the existing bodies p > 2, p != b, in the 27 cells around its own
// (the cell relation is symmetric, the reference's index aliasing included),
// and the sum over them is taken in any fixed order.  The three cells of a row
// (x - 1, x, x + 1) are consecutive linear indices, hence one contiguous range
// of the cell-sorted bodies: a body walks 9 ranges.  The warp's bodies queue
// their partners (record positions, per lane in shared memory) during the
// walk; then the warp evaluates the queued pair terms 32 at a time, every lane
// busy whatever the lengths of the bodies' lists.  A round's terms of one body
// sit in adjacent lanes: a segmented scan over the warp (five shuffle steps)
// leaves each list's sum in its last lane, which the body adds to its own sums
// (a fixed order: deterministic).  The pair term is FP64 with one
// reciprocal square root (G m dx / D^3 = G m dx (1/D)^3); against the exact
// mode, only its rounding and the order of the sum differ.
constexpr int FGW = 4;   // warps per block
constexpr int FGQ = 32;  // queued partners per lane and round

// The partner at position q against a body at (xb, yb, zb) of radius Rb: the
// partner's x, y, z and partner mass in two 16-byte loads of the compact gp
// array (a zero mass for bodies that add no term), its radius from its record.
__device__ __forceinline__ void term_fast(double xb, double yb, double zb, double Rb, const double4 *__restrict__ gp,
                                          const GRec *__restrict__ grec, int q, const MGArgs &A, double &tx,
                                          double &ty, double &tz)
{
      const double2 *r = reinterpret_cast<const double2 *>(gp + q);
      const double2 xy = r[0], zm = r[1];
      const double dx = xy.x - xb, dy = xy.y - yb, dz = zm.x - zb;
      double r2 = dx * dx + dy * dy + dz * dz;
      if (A.soft) {
            const double s = A.sp * (Rb + grec[q].R);
            r2 += s * s;
      }
      const double ri = rsqrt(r2);
      const double w = A.G * zm.y * (ri * ri * ri);
      tx = w * dx;
      ty = w * dy;
      tz = w * dz;
}

__global__ void __launch_bounds__(FGW * 32, 8) k_mesh_grav_fast(DevState S, MGArgs A, const uint32_t *__restrict__ keys,
                                                               const int *__restrict__ vals,
                                                               const int2 *__restrict__ crange,
                                                               const GRec *__restrict__ grec,
                                                               const double4 *__restrict__ gp, double *__restrict__ ax,
                                                               double *__restrict__ ay, double *__restrict__ az,
                                                               double *__restrict__ terms, long N,
                                                               double *__restrict__ cpart)
{
      __shared__ int qb[FGW][32 * FGQ];
      __shared__ unsigned char owner[FGW][32 * FGQ];
      __shared__ int pre[FGW][32];
      __shared__ double csum[12][FGW];
      const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
      const int t = blockIdx.x * blockDim.x + threadIdx.x;  // cell order
      const int t0 = t - lane;                               // the warp's first record
      const bool act = t <= A.lid;
      const int b = act ? vals[t] : 0;
      GRec me;
      me.x = me.y = me.z = me.m = me.R = 0.;
      me.ex = 0;
      if (act) me = grec[t];
      double a_x = 0., a_y = 0., a_z = 0.;
      bool walk = false;
      {
            // the bodies' terms of the 12 chains (bodies 0..2, CM_acc), summed over
            // the block in a fixed shape: cpart[12 block + chain]
            double tv[12];
            if (act) {
                  walk = body_prologue(S, A, me, b, t, terms, N, ax, ay, az, a_x, a_y, a_z, tv) && A.mutual;
            } else {
                  for (int c = 0; c < 12; c++) tv[c] = 0.;
            }
            for (int c = 0; c < 12; c++) {
                  double v = tv[c];
                  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                  if (lane == 0) csum[c][w] = v;
            }
            __syncthreads();
            if (threadIdx.x < 12) {
                  double v = 0.;
                  for (int q = 0; q < FGW; q++) v += csum[threadIdx.x][q];
                  cpart[12 * (size_t)blockIdx.x + threadIdx.x] = v;
            }
      }
      const uint32_t L = act ? keys[t] : 0xffffffffu;
      walk = walk && L != 0xffffffffu;  // outside the collision cube: no pairs
      const long long dd = (long long)A.d * A.d;
      int skip = 0;
      bool more = walk;
      while (__any_sync(0xffffffffu, more)) {
            int cnt = 0;
            if (more) {
                  int idx = 0;
#pragma unroll 1
                  for (int r = 0; r < 9; ++r) {
                        int s0, e0;
                        if (!row_range(crange, d_row(L, r, A.d, dd), A.cell_cap, &s0, &e0)) continue;
                        for (int q = s0; q < e0; ++q) {
                              if (q == t) continue;  // (bodies 0..2 and removed ones add zero terms)
                              if (idx >= skip && idx < skip + FGQ) qb[w][lane * FGQ + idx - skip] = q;
                              ++idx;
                        }
                  }
                  cnt = min(idx - skip, FGQ);
                  more = idx > skip + FGQ;
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
                  double tx = 0., ty = 0., tz = 0.;
                  int a = lane;  // the lane where this entry's list starts in the round
                  if (fi < total) {
                        const int o = owner[w][fi];
                        const int q = qb[w][o * FGQ + fi - pre[w][o]];
                        const double2 *ow = reinterpret_cast<const double2 *>(grec + t0 + o);
                        const double2 oxy = ow[0], oz = ow[1];
                        term_fast(oxy.x, oxy.y, oz.x, A.soft ? grec[t0 + o].R : 0., gp, grec, q, A, tx, ty, tz);
                        a = max(pre[w][o] - f0, 0);
                  }
                  // segmented inclusive scan over the round (the lists are contiguous in
                  // lane order): the last lane of a list then holds the list's sum
#pragma unroll
                  for (int dl = 1; dl < 32; dl <<= 1) {
                        const double ux = __shfl_up_sync(0xffffffffu, tx, dl);
                        const double uy = __shfl_up_sync(0xffffffffu, ty, dl);
                        const double uz = __shfl_up_sync(0xffffffffu, tz, dl);
                        if (lane - dl >= a) {
                              tx += ux;
                              ty += uy;
                              tz += uz;
                        }
                  }
                  // each body takes its list's sum of this round from the list's last lane
                  const int i0 = max(mine, f0), i1 = min(mine + cnt, f0 + 32);
                  const int src = i1 > i0 ? i1 - 1 - f0 : lane;
                  const double sx = __shfl_sync(0xffffffffu, tx, src);
                  const double sy = __shfl_sync(0xffffffffu, ty, src);
                  const double sz = __shfl_sync(0xffffffffu, tz, src);
                  if (i1 > i0) {
                        a_x += sx;
                        a_y += sy;
                        a_z += sz;
                  }
            }
            __syncwarp();
            skip += FGQ;
      }
      if (walk || (act && me.ex && b > 2)) {
            ax[b] = a_x; ay[b] = a_y; az[b] = a_z;
      }
}

// Bodies 0..2 and CM_acc.  Chain w (0..8: body w/3, component w%3; 9..11:
// CM_acc components) sums its terms in slot order.  exact: one CTA (one warp)
// per chain staging the terms through shared memory (warp_chain_sum), so the
// FP64 sum is the reference's sequential one (a body that does not exist adds
// +0.0, which leaves any sum other than -0.0 unchanged).  Body i's chain starts
// from its central term, CM_acc from 0.
__device__ __forceinline__ double chain_init(int w, const double *ax, const double *ay, const double *az)
{
      if (w >= 9) return 0.;
      int i = w / 3, comp = w % 3;
      return comp == 0 ? ax[i] : comp == 1 ? ay[i] : az[i];
}

__device__ __forceinline__ bool chain_live(int w, const DevState &S, const MGArgs &A)
{
      return w >= 9 ? A.central : (S.ex[w / 3] && A.mutual);
}

__global__ void __launch_bounds__(32) k_mesh_chains(DevState S, MGArgs A, const double *__restrict__ terms, long N,
                                                    const double *__restrict__ ax, const double *__restrict__ ay,
                                                    const double *__restrict__ az, double *__restrict__ tot)
{
      __shared__ __align__(16) double stage[CHN];
      const int w = blockIdx.x;  // one chain per CTA
      double s = chain_init(w, ax, ay, az);
      if (chain_live(w, S, A)) {
            const int k0 = w >= 9 ? 0 : 3;
            const double *t =
                w >= 9 ? cm_chain(const_cast<double *>(terms), A, N, w - 9) : terms + (size_t)w * N + k0;
            const long n = w >= 9 ? (long)(A.j2.on ? 2 : 1) * (A.lid + 1) : (long)A.lid + 1 - k0;
            s = warp_chain_sum(t, n > 0 ? n : 0, s, stage);
      }
      if (threadIdx.x == 0) tot[w] = s;
}

// Non-exact modes: deterministic two-level sums of the same 12 chains.
constexpr int RB12 = 256;
__global__ void k_mesh_chains_part(DevState S, MGArgs A, const double *__restrict__ terms, long N,
                                   double *__restrict__ part)
{
      __shared__ double sh[12][RB12 / 32];
      double s[12];
      for (int w = 0; w < 12; w++) s[w] = 0.;
      const int n = A.lid + 1;
      const int f = A.j2.on ? 2 : 1;
      for (int k = blockIdx.x * RB12 + threadIdx.x; k < n; k += gridDim.x * RB12) {
            if (A.cellterms) {  // cell order: every position holds its terms (zeros for empty slots and bodies 0..2)
                  for (int w = 0; w < 9; w++) s[w] += terms[(size_t)w * N + k];
            } else {
                  if (!S.ex[k]) continue;
                  for (int w = 0; w < 9; w++)
                        if (k >= 3) s[w] += terms[(size_t)w * N + k];
            }
            for (int c = 0; c < 3; c++) {
                  const double *t = cm_chain(const_cast<double *>(terms), A, N, c) + (size_t)f * k;
                  s[9 + c] += f == 2 ? t[0] + t[1] : t[0];
            }
      }
      const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
      for (int w = 0; w < 12; w++) {
            double v = s[w];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) sh[w][wp] = v;
      }
      __syncthreads();
      if (threadIdx.x < 12) {
            double v = 0.;
            for (int q = 0; q < RB12 / 32; q++) v += sh[threadIdx.x][q];
            part[blockIdx.x * 12 + threadIdx.x] = v;
      }
}

// The block partials folded in a fixed shape (deterministic): thread i of
// CHF (a multiple of 12) takes chain i % 12 of partials i / 12, i / 12 + CHF / 12,
// ... -- consecutive threads read consecutive doubles -- and each chain's
// CHF / 12 sums are added in order.
constexpr int CHF = 768;
__global__ void __launch_bounds__(CHF) k_mesh_chains_fold(DevState S, MGArgs A, const double *__restrict__ part,
                                                         int nparts, const double *__restrict__ ax,
                                                         const double *__restrict__ ay, const double *__restrict__ az,
                                                         double *__restrict__ tot)
{
      constexpr int L = CHF / 12;
      __shared__ double sh[12][L];
      const int i = threadIdx.x, w = i % 12, l = i / 12;
      double s = 0.;
      for (int b = l; b < nparts; b += L) s += part[12 * (size_t)b + w];
      sh[w][l] = s;
      __syncthreads();
      if (i < 12) {
            double v = 0.;
            for (int q = 0; q < L; q++) v += sh[i][q];
            tot[i] = chain_live(i, S, A) ? chain_init(i, ax, ay, az) + v : chain_init(i, ax, ay, az);
      }
}

// CM_acc and bodies 0..2: chain totals, then the (0,1), (0,2), (1,2) pairs
// (src/physics.c:297-341).
__global__ void k_mesh_big3(DevState S, MGArgs A, const double *__restrict__ tot, double *ax, double *ay, double *az,
                            double *cm_acc)
{
      if (threadIdx.x != 0) return;
      if (A.central) {
            cm_acc[0] = tot[9]; cm_acc[1] = tot[10]; cm_acc[2] = tot[11];
      } else {
            cm_acc[0] = cm_acc[1] = cm_acc[2] = 0.;
      }
      double a[3][3];
      for (int i = 0; i < 3; i++) {
            if (!S.ex[i]) continue;
            a[i][0] = tot[3 * i];
            a[i][1] = tot[3 * i + 1];
            a[i][2] = tot[3 * i + 2];
      }
      if (A.mutual) {
            const int pr[3][2] = {{0, 1}, {0, 2}, {1, 2}};
            for (int q = 0; q < 3; q++) {
                  int u = pr[q][0], w = pr[q][1];
                  if (!(S.ex[u] && S.ex[w])) continue;
                  pair_add(S, u, w, A.G, A.sp, A.soft, a[u][0], a[u][1], a[u][2]);
                  pair_add(S, w, u, A.G, A.sp, A.soft, a[w][0], a[w][1], a[w][2]);
            }
      }
      for (int i = 0; i < 3; i++) {
            if (!S.ex[i]) continue;
            ax[i] = a[i][0]; ay[i] = a[i][1]; az[i] = a[i][2];
      }
}

}  // namespace

int three_largest_state(int *idx)
{
      Ctx &c = ctx();
      cudaStream_t st = c.s;
      const int lid = c.largest_id;
      DevState S = dev_state();
      int *first3 = c.n_dev + 2, *out = c.n_dev + 5;
      k_first3<<<1, 32, 0, st>>>(c.ex, lid, first3);
      NCG_LAUNCHED();
      const int np = std::min(256, std::max(1, (lid + 1 + TB - 1) / TB));
      double *partR = c.red + 1024;
      int *parti = (int *)(c.red + 1792);
      k_top3_part<<<np, TB, 0, st>>>(S, lid, first3, partR, parti);
      NCG_LAUNCHED();
      k_top3_final<<<1, 32, 0, st>>>(S, first3, partR, parti, np, c.P.par_mesh_bool, out);
      NCG_LAUNCHED();
      if (idx) {  // (the loop itself needs no indices on the host)
            NCG_CK(cudaMemcpyAsync(idx, out, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
            NCG_CK(cudaStreamSynchronize(st));
      }
      return NCGPU_OK;
}

// vector_field in mesh mode on the device state; acc blocks + cm_acc.
int mesh_gravity_state(const J2Arg &j2)
{
      Ctx &c = ctx();
      cudaStream_t st = c.s;
      const int lid = c.largest_id;
      const long N = c.n_max;
      constexpr int MAXP = 1184;  // block partials of the parallel chain sums (8 per SM)
      // (fast kernel: its blocks' chain sums after the terms' room)
      const int nfast = lid >= 0 ? (lid + FGW * 32) / (FGW * 32) : 1;
      NCG_TRY(ensure_partial((size_t)(j2.on ? 15 : 12) * N + 12 * (size_t)std::max(MAXP, nfast)));
      double *cpart = c.partial + (size_t)(j2.on ? 15 : 12) * N;
      bool fast_done = false;
      DevState S = dev_state();
      MGArgs A{lid, c.P.par_collision_cube_cells, c.P.par_central_mass_bool, c.P.par_mutual_bool,
               c.P.par_softening_parameter != 0., (long long)c.cell_cap, c.P.par_G, c.P.par_softening_parameter,
               c.cm,
               c.mesh_valid ? c.mesh_n - 1 : -1, c.P.par_N_tilde, c.mesh_nfev, c.evx, c.fev,
               c.mesh_nfev > 0 ? c.xhead : nullptr, c.mesh_valid ? c.mesh_nvis : 0, c.vis, c.cand_p, j2,
               c.P.par_gravity_mode != NCGPU_GRAVITY_EXACT};
      double *ax = c.acc, *ay = c.acc + N, *az = c.acc + 2 * N;
      if (lid >= 0) {
            GRec *grec = (GRec *)c.mrec;
            double4 *gp = (double4 *)c.gpart;
            // the fast modes' order-free kernel where a body's pairs are exactly its
            // 27-cell neighbours (no big bodies' visits, no fragments appended)
            const bool fast = A.cellterms && c.mesh_valid && A.nvis == 0 && A.nfev == 0 && lid == A.lid0;
            if (c.mesh_valid) {
                  k_grav_records<<<(c.mesh_n + 255) / 256, 256, 0, st>>>(S, c.mvals, c.mesh_n, grec,
                                                                         fast ? gp : nullptr);
                  NCG_LAUNCHED();
            }
            fast_done = fast;
            if (fast)
                  k_mesh_grav_fast<<<nfast, FGW * 32, 0, st>>>(S, A, c.mkeys, c.mvals, c.crange, grec, gp, ax, ay, az,
                                                               c.partial, N, cpart);
            else
                  k_mesh_grav<<<(lid + 256) / 256, 256, 0, st>>>(S, A, c.ckey, c.mkeys, c.mvals, c.crange, c.mesh_valid,
                                                                grec, ax, ay, az, c.partial, N);
            NCG_LAUNCHED();
      }
      double *tot = c.red + 3584;
      if (c.P.par_gravity_mode == NCGPU_GRAVITY_EXACT) {
            k_mesh_chains<<<12, 32, 0, st>>>(S, A, c.partial, N, ax, ay, az, tot);
            NCG_LAUNCHED();
      } else if (fast_done) {  // the fast kernel's block sums
            k_mesh_chains_fold<<<1, CHF, 0, st>>>(S, A, cpart, nfast, ax, ay, az, tot);
            NCG_LAUNCHED();
      } else {
            const int np = std::min(MAXP, std::max(1, (lid + RB12) / RB12));
            k_mesh_chains_part<<<np, RB12, 0, st>>>(S, A, c.partial, N, cpart);
            NCG_LAUNCHED();
            k_mesh_chains_fold<<<1, CHF, 0, st>>>(S, A, cpart, np, ax, ay, az, tot);
            NCG_LAUNCHED();
      }
      k_mesh_big3<<<1, 32, 0, st>>>(S, A, tot, ax, ay, az, c.cm_acc);
      NCG_LAUNCHED();
      return NCGPU_OK;
}

}  // namespace ncg

using namespace ncg;

extern "C" int ncgpu_three_largest(int *idx)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      NCG_TRY(three_largest_state(idx));
      return sync_scalars();
}
