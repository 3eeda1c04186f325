// Shared internals of libncgpu: the device-resident context, error plumbing
// and small device helpers.  Host code is single-threaded by contract (the
// reference itself is a single-threaded program with global state).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include "../../include/ncgpu.h"

namespace ncg {

// Records a CUDA failure (text kept for ncgpu_last_error) and returns the
// library status.
int cuda_fail(cudaError_t e, const char *what, const char *file, int line);
void note_launch();          // counts kernel launches of the current API call
void reset_launches();
int launches();

#define NCG_CK(call)                                                          \
      do {                                                                    \
            cudaError_t e_ = (call);                                          \
            if (e_ != cudaSuccess) return ncg::cuda_fail(e_, #call, __FILE__, __LINE__); \
      } while (0)

// After a <<<>>> launch: count it and surface launch-configuration errors.
#define NCG_LAUNCHED()                                                        \
      do {                                                                    \
            ncg::note_launch();                                               \
            cudaError_t e_ = cudaGetLastError();                              \
            if (e_ != cudaSuccess) return ncg::cuda_fail(e_, "kernel launch", __FILE__, __LINE__); \
      } while (0)

#define NCG_TRY(call)                                                         \
      do {                                                                    \
            int s_ = (call);                                                  \
            if (s_ != NCGPU_OK) return s_;                                    \
      } while (0)

// Strided read-only view of body fields: AoS (struct moonlet, stride 8) or
// SoA (stride 1).
struct BodyView {
      const double *x, *y, *z, *vx, *vy, *vz, *m, *R;
      long stride;
      const int *ex;
};

// The J2 term of a force evaluation (src/physics.c:149-160): off, or on with
// R_unit, the J2 in force and the central mass M.
struct J2Arg {
      int on;
      double R, J2, M;
};

// J2_value when it is nonzero, else the fluid-body J2 of central mass M and
// sideral rotation omega, the expression of src/structure.c:507 and
// src/rk4.c:462 in its order.
inline double j2_value(const ncgpu_params &P, double M, double omega)
{
      if (P.par_J2 != 0.) return P.par_J2;
      return 0.5 * omega * omega * P.par_R_unit * P.par_R_unit * P.par_R_unit / (P.par_G * M);
}

// The J2 term of a force evaluation with the J2 value j2 (central mass M).
inline J2Arg j2_arg(const ncgpu_params &P, double M, double j2)
{
      return J2Arg{P.par_J2_bool && P.par_central_mass_bool, P.par_R_unit, j2, M};
}

// Adds body k's J2 term to its acceleration a[] and returns CM_acc's share in
// c[], every operation the reference's in its order with IEEE rounding:
//   r2 = rk*rk, r5 = r3*r2, K = mu*R*R*J2/r5, q = 7.5/r2*DZ*DZ
//   a += K*(-1.5*DX + q*DX), K*(-1.5*DY + q*DY), K*(-4.5*DZ + q*DZ)
//   c  = K*(1.5*DX - q*DX)*mk/M, ... (4.5 for z)
__device__ __forceinline__ void d_j2(const J2Arg &j, double mu, double DX, double DY, double DZ, double rk,
                                     double r3, double mk, double &ax, double &ay, double &az, double *c)
{
      const double r2 = __dmul_rn(rk, rk);
      const double r5 = __dmul_rn(r3, r2);
      const double K = __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(mu, j.R), j.R), j.J2), r5);
      const double q = __dmul_rn(__dmul_rn(__ddiv_rn(7.5, r2), DZ), DZ);
      const double qx = __dmul_rn(q, DX), qy = __dmul_rn(q, DY), qz = __dmul_rn(q, DZ);
      ax = __dadd_rn(ax, __dmul_rn(K, __dadd_rn(__dmul_rn(-1.5, DX), qx)));
      ay = __dadd_rn(ay, __dmul_rn(K, __dadd_rn(__dmul_rn(-1.5, DY), qy)));
      az = __dadd_rn(az, __dmul_rn(K, __dadd_rn(__dmul_rn(-4.5, DZ), qz)));
      c[0] = __ddiv_rn(__dmul_rn(__dmul_rn(K, __dsub_rn(__dmul_rn(1.5, DX), qx)), mk), j.M);
      c[1] = __ddiv_rn(__dmul_rn(__dmul_rn(K, __dsub_rn(__dmul_rn(1.5, DY), qy)), mk), j.M);
      c[2] = __ddiv_rn(__dmul_rn(__dmul_rn(K, __dsub_rn(__dmul_rn(4.5, DZ), qz)), mk), j.M);
}

// x / b correctly rounded (round to nearest even) from y = RN(1/b), with
// Markstein's residual correction (P. Markstein, IBM J. Res. Dev. 34 (1990)
// 111-119; J.-M. Muller et al., Handbook of Floating-Point Arithmetic, ch. 4)
// applied twice: r = x - b q is exact when q is within an ulp of x/b, and then
// RN(q + r y) = RN(x/b); the first correction brings RN(x y) within that ulp.
// Valid for finite nonzero b with the quotient and residuals in the normal
// range; a zero x gives x * y, a zero with the quotient's sign.  A short
// dependent chain (one multiply, four FMAs) for the latency-bound recurrences
// that need the quotient; the reciprocal is computed off the chain.
__device__ __forceinline__ double div_by_recip(double x, double b, double y)
{
      if (x == 0.) return __dmul_rn(x, y);
      double q = __dmul_rn(x, y);
      double r = __fma_rn(-q, b, x);
      q = __fma_rn(r, y, q);
      r = __fma_rn(-q, b, x);
      return __fma_rn(r, y, q);
}

// FP32 reciprocal square root (MUFU, flush-to-zero) and sm_100a's packed
// f32x2 arithmetic (one instruction on both halves of a 64-bit register pair).
__device__ __forceinline__ float rsqrt_ftz(float x)
{
      float y;
      asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
      return y;
}

// Packed pairs of FP32 values (sm_100a f32x2 arithmetic: one instruction
// operates on both halves).
typedef unsigned long long f2;

__device__ __forceinline__ f2 f2_pack(float lo, float hi)
{
      f2 r;
      asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
      return r;
}
__device__ __forceinline__ void f2_unpack(f2 v, float &lo, float &hi)
{
      asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2 f2_sub(f2 a, f2 b)
{
      f2 r;
      asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
      return r;
}
__device__ __forceinline__ f2 f2_add(f2 a, f2 b)
{
      f2 r;
      asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
      return r;
}
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b)
{
      f2 r;
      asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
      return r;
}
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c)
{
      f2 r;
      asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
      return r;
}
__device__ __forceinline__ f2 f2_rsqrt(f2 q)
{
      float lo, hi;
      f2_unpack(q, lo, hi);
      return f2_pack(rsqrt_ftz(lo), rsqrt_ftz(hi));
}

// Two tiles' boxes (centre xyz, half extents xyz) are near when the gap
// between them is below theta times the larger full diagonal.
__device__ __forceinline__ bool tiles_near(const double *__restrict__ bi, const double *__restrict__ bj, double theta)
{
      double g2 = 0., di = 0., dj = 0.;
      for (int d = 0; d < 3; d++) {
            double gap = fabs(bi[d] - bj[d]) - bi[3 + d] - bj[3 + d];
            if (gap > 0.) g2 += gap * gap;
            di += bi[3 + d] * bi[3 + d];
            dj += bj[3 + d] * bj[3 + d];
      }
      double dmax2 = 4. * fmax(di, dj);  // squared full diagonal
      return g2 < theta * theta * dmax2;
}

// The 27 neighbour cells of a cell L (linear index i + j d + k d^2) as 9 rows
// of three consecutive indices (x - 1, x, x + 1): row r (0..8) is centred on
// L + (r % 3 - 1) d + (r / 3 - 1) d^2, so the cell slots l = 26..0 of the
// reference's pop order are the rows r = 8..0, each from x + 1 down to x - 1.
__device__ __forceinline__ long long d_row(long long L, int r, int d, long long dd)
{
      return L + (r % 3 - 1) * (long long)d + (r / 3 - 1) * dd;
}

// The [first, end) ranges of the cells mid - 1, mid, mid + 1 in the cell table
// ({-1, -1} for an empty cell or one outside [0, cap)); three independent loads.
__device__ __forceinline__ void row_cells(const int2 *__restrict__ crange, long long mid, long long cap, int2 (&cr)[3])
{
#pragma unroll
      for (int x = 0; x < 3; ++x) {
            const long long c = mid - 1 + x;
            cr[x] = (c >= 0 && c < cap) ? crange[c] : make_int2(-1, -1);
      }
}

// The row's cells are consecutive keys, hence one contiguous range [s, e) of
// the cell-sorted bodies; false when all three are empty.
__device__ __forceinline__ bool row_range(const int2 *__restrict__ crange, long long mid, long long cap, int *s, int *e)
{
      int2 cr[3];
      row_cells(crange, mid, cap, cr);
      const int s0 = cr[0].x >= 0 ? cr[0].x : cr[1].x >= 0 ? cr[1].x : cr[2].x;
      if (s0 < 0) return false;
      *s = s0;
      *e = cr[2].y >= 0 ? cr[2].y : cr[1].y >= 0 ? cr[1].y : cr[0].y;
      return true;
}


// Sequential FP64 sum s + t[0] + t[1] + ... + t[n-1], in that order with IEEE
// rounding, by one warp (the result is lane 0's): the lanes stage CHN terms at
// a time in shared memory (`stage`, CHN doubles, 16-byte aligned) with
// coalesced loads, the next block in flight while lane 0 adds, two terms per
// shared load.  Launched as one warp per CTA, so that every chain has an SM's
// FP64 pipe to itself.
constexpr int CHN = 512;
__device__ __forceinline__ double warp_chain_sum(const double *__restrict__ t, long n, double s, double *stage)
{
      const int lane = threadIdx.x & 31;
      double v[CHN / 32];
#pragma unroll
      for (int u = 0; u < CHN / 32; u++) {
            const long k = (long)u * 32 + lane;
            v[u] = k < n ? t[k] : 0.;
      }
      for (long base = 0; base < n; base += CHN) {
#pragma unroll
            for (int u = 0; u < CHN / 32; u++) stage[u * 32 + lane] = v[u];
            __syncwarp();
#pragma unroll
            for (int u = 0; u < CHN / 32; u++) {  // the next block, in flight during the sums
                  const long k = base + CHN + (long)u * 32 + lane;
                  v[u] = k < n ? t[k] : 0.;
            }
            if (lane == 0) {
                  const long m = n - base < CHN ? n - base : CHN;
                  if (m == CHN) {  // full block: fixed trip count
                        const double2 *st2 = reinterpret_cast<const double2 *>(stage);
#pragma unroll 16
                        for (int q = 0; q < CHN / 2; q++) {
                              const double2 pr = st2[q];
                              s = __dadd_rn(s, pr.x);
                              s = __dadd_rn(s, pr.y);
                        }
                  } else {
                        for (int q = 0; q < m; q++) s = __dadd_rn(s, stage[q]);
                  }
            }
            __syncwarp();
      }
      return s;
}


// The same sum, taking whole runs of terms at once (display()'s total mass of
// up to millions of positive masses).  While the running sum is a normal number
// of binade e (|s| in [2^e, 2^(e+1))) it is an integer multiple T of
// u = 2^(e-52), and s + x rounds to (T + R)u, R the integer nearest x/u, as
// long as T + R stays inside the binade with a unit to spare
// (2^52 < |T + R| < 2^53, or |T + R| = 2^52 with x/u - R pointing away from
// zero) and x/u is not an odd multiple of 1/2 (a tie, whose rounding would
// depend on T's last bit).  So terms are rounded to the spacing independently
// and their integer prefix sums checked against the binade.
//
// A block of RUN_NW warps takes RUN_NW windows of RUN_W terms a round: each
// warp stages its window in shared memory (lane L's RUN_Q consecutive terms in
// row L) and sums it for the binade the round starts in, with the range of its
// prefix sums; warp 0 then accepts the windows in order while they keep the
// sum inside the binade, and walks the first one that does not term by term
// (run_window: every term before the first that breaks a condition taken at
// once, that term -- a binade change, a tie, a NaN or an infinity, a term of
// 2^47 units or more, a sum that is zero, subnormal or beyond 2^+-969 -- added
// by itself, and the pass resumed after it; after a short run the next
// SEQ_RUN terms go one by one).  The next round starts after that window.
// Sums whose running value keeps changing binade (zero-mean terms) gain
// nothing, so the other reference-order sums keep warp_chain_sum.
constexpr int RUN_Q = 16, RUN_NW = 16, RUN_W = 32 * RUN_Q;
constexpr int RUN_ROW = RUN_Q + 1;                  // padded row: conflict-free transposed reads
constexpr int RUN_STAGE = RUN_NW * 32 * RUN_ROW;    // doubles of dynamic shared memory
constexpr int SEQ_SHORT = 64, SEQ_RUN = 256;
constexpr double SEQ_MAG = 6755399441055744.0;  // 1.5 * 2^52: adding it rounds |q| < 2^51 to an integer

struct SeqBin {
      long long T;  // s = T * u
      double u, inv;
      bool ok;
};

__device__ __forceinline__ SeqBin seq_bin(double s)
{
      SeqBin b;
      const unsigned long long w = (unsigned long long)__double_as_longlong(s);
      const int ef = (int)((w >> 52) & 0x7ff);
      b.ok = ef >= 54 && ef <= 2023;  // u = 2^(ef-1075) and 1/u both normal
      const long long M = (long long)((w & 0xfffffffffffffull) | 0x10000000000000ull);
      b.T = (w >> 63) ? -M : M;
      b.u = __longlong_as_double((long long)((unsigned long long)(unsigned)(ef - 52) << 52));
      b.inv = __longlong_as_double((long long)((unsigned long long)(unsigned)(2098 - ef) << 52));
      return b;
}

__device__ __forceinline__ double run_term(const double *buf, int p)
{
      return buf[(p / RUN_Q) * RUN_ROW + p % RUN_Q];
}

// One warp walks window buf (terms 0 .. wl-1) from term o on, from the sum s.
__device__ __forceinline__ double run_window(const double *buf, int o, int wl, double s)
{
      const int lane = threadIdx.x & 31, p0 = lane * RUN_Q;
      SeqBin b = seq_bin(s);
      while (o < wl) {
            if (!b.ok) {  // no binade: the next term by itself
                  s = __dadd_rn(s, run_term(buf, o));
                  o++;
                  b = seq_bin(s);
                  continue;
            }
            const bool pos = b.T > 0;
            double acc = 0., mn = 0., mx = 0., P[RUN_Q];
            unsigned bad = 0u, dok = 0u;
#pragma unroll
            for (int j = 0; j < RUN_Q; j++) {
                  const double x = buf[lane * RUN_ROW + j];
                  const bool live = p0 + j >= o && p0 + j < wl;
                  const double y = __fma_rn(x, b.inv, SEQ_MAG);
                  const double r = __dsub_rn(y, SEQ_MAG);  // x/u rounded (exact while |x/u| < 2^51)
                  const double d = __fma_rn(x, b.inv, -r);  // x/u - r, exact
                  const bool good = fabs(r) < 0x1p47 && fabs(d) != 0.5;
                  acc = __dadd_rn(acc, live && good ? r : 0.);  // integers below 2^52: exact
                  P[j] = acc;
                  mn = fmin(mn, acc);
                  mx = fmax(mx, acc);
                  bad |= (unsigned)(live && !good) << j;
                  dok |= (unsigned)(pos ? d >= 0. : d <= 0.) << j;
            }
            const long long tot = __double2ll_rn(acc);
            long long inc = tot;
#pragma unroll
            for (int k = 1; k < 32; k <<= 1) {
                  const long long v = __shfl_up_sync(0xffffffffu, inc, k);
                  if (lane >= k) inc += v;
            }
            const long long T0 = b.T + (inc - tot);  // the sum before this lane's terms
            const long long wsum = __shfl_sync(0xffffffffu, inc, 31);
            const long long LO1 = pos ? (1LL << 52) + 1 : -((1LL << 53) - 1);
            const long long HI1 = pos ? (1LL << 53) - 1 : -((1LL << 52) + 1);
            const bool lane_ok = !bad && T0 + __double2ll_rn(mn) >= LO1 && T0 + __double2ll_rn(mx) <= HI1;
            if (__all_sync(0xffffffffu, lane_ok)) {  // the rest of the window
                  s = __dmul_rn(__ll2double_rn(b.T + wsum), b.u);
                  break;
            }
            // the first term that breaks a condition, and the sum before it
            const long long LOe = pos ? (1LL << 52) : -((1LL << 53) - 1);
            const long long HIe = pos ? (1LL << 53) - 1 : -(1LL << 52);
            const long long EDGE = pos ? LOe : HIe;
            int jf = RUN_Q;
#pragma unroll
            for (int j = RUN_Q - 1; j >= 0; j--) {
                  const bool live = p0 + j >= o && p0 + j < wl;
                  const long long Tj = T0 + __double2ll_rn(P[j]);
                  const bool brk = live && (((bad >> j) & 1u) || Tj < LOe || Tj > HIe ||
                                            (Tj == EDGE && !((dok >> j) & 1u)));
                  jf = brk ? j : jf;
            }
            long long Tb = T0;
#pragma unroll
            for (int j = 0; j < RUN_Q - 1; j++) Tb = j + 1 == jf ? T0 + __double2ll_rn(P[j]) : Tb;
            const unsigned bm = __ballot_sync(0xffffffffu, jf < RUN_Q);
            if (!bm) {
                  s = __dmul_rn(__ll2double_rn(b.T + wsum), b.u);
                  break;
            }
            const int lf = __ffs(bm) - 1;
            const int pf = lf * RUN_Q + __shfl_sync(0xffffffffu, jf, lf);
            s = __dmul_rn(__ll2double_rn(__shfl_sync(0xffffffffu, Tb, lf)), b.u);
            s = __dadd_rn(s, run_term(buf, pf));
            const int taken = pf - o;
            o = pf + 1;
            if (taken < SEQ_SHORT) {
                  const int e = wl < o + SEQ_RUN ? wl : o + SEQ_RUN;
                  for (; o < e; o++) s = __dadd_rn(s, run_term(buf, o));
            }
            b = seq_bin(s);
      }
      return s;
}

// A window's integer sum at the spacing of binade b, the range of its prefix
// sums (the empty prefix included) and whether a term cannot be taken.
struct RunPart {
      long long tot, mn, mx;
      int bad;
};

__device__ __forceinline__ RunPart run_part(const double *buf, int wl, const SeqBin &b)
{
      const int lane = threadIdx.x & 31, p0 = lane * RUN_Q;
      double acc = 0., mn = 0., mx = 0.;
      bool bad = false;
#pragma unroll
      for (int j = 0; j < RUN_Q; j++) {
            const double x = buf[lane * RUN_ROW + j];
            const bool live = p0 + j < wl;
            const double y = __fma_rn(x, b.inv, SEQ_MAG);
            const double r = __dsub_rn(y, SEQ_MAG);
            const double d = __fma_rn(x, b.inv, -r);
            const bool good = fabs(r) < 0x1p47 && fabs(d) != 0.5;
            acc = __dadd_rn(acc, live && good ? r : 0.);
            mn = fmin(mn, acc);
            mx = fmax(mx, acc);
            bad |= live && !good;
      }
      const long long tot = __double2ll_rn(acc);
      long long inc = tot;
#pragma unroll
      for (int k = 1; k < 32; k <<= 1) {
            const long long v = __shfl_up_sync(0xffffffffu, inc, k);
            if (lane >= k) inc += v;
      }
      long long lo = inc - tot + __double2ll_rn(mn), hi = inc - tot + __double2ll_rn(mx);
#pragma unroll
      for (int k = 16; k > 0; k >>= 1) {
            const long long a = __shfl_xor_sync(0xffffffffu, lo, k), c = __shfl_xor_sync(0xffffffffu, hi, k);
            lo = a < lo ? a : lo;
            hi = c > hi ? c : hi;
      }
      RunPart r;
      r.tot = __shfl_sync(0xffffffffu, inc, 31);
      r.mn = lo;
      r.mx = hi;
      r.bad = __any_sync(0xffffffffu, bad);
      return r;
}

// s + t[0] + ... + t[n-1] by the whole block (RUN_NW warps; every thread
// returns it); stage: RUN_STAGE doubles of shared memory.
__device__ __forceinline__ double block_run_sum(const double *__restrict__ t, long n, double s, double *stage)
{
      __shared__ RunPart part[RUN_NW];
      __shared__ double sh_s;
      __shared__ long sh_pos;
      const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
      double *buf = stage + w * 32 * RUN_ROW;
      long pos = 0;
      while (pos < n) {
            const SeqBin b = seq_bin(s);
            const long start = pos + (long)w * RUN_W;
            const long left = n - start;
            const int wl = left <= 0 ? 0 : left < RUN_W ? (int)left : RUN_W;
#pragma unroll 4
            for (int i = 0; i < RUN_Q; i++) {  // window term i*32 + lane: row (i*32 + lane) / RUN_Q
                  const int p = i * 32 + lane;
                  buf[(p / RUN_Q) * RUN_ROW + p % RUN_Q] = p < wl ? t[start + p] : 0.;
            }
            __syncwarp();
            RunPart r{0, 0, 0, 0};
            if (b.ok && wl > 0) r = run_part(buf, wl, b);
            if (lane == 0) part[w] = r;
            __syncthreads();
            if (w == 0) {
                  double s2 = s;
                  long p2;
                  if (b.ok) {
                        const bool pos_s = b.T > 0;
                        const long long LO1 = pos_s ? (1LL << 52) + 1 : -((1LL << 53) - 1);
                        const long long HI1 = pos_s ? (1LL << 53) - 1 : -((1LL << 52) + 1);
                        long long T = b.T;
                        int k = 0;
                        for (; k < RUN_NW && pos + (long)k * RUN_W < n; k++) {  // windows taken whole
                              const RunPart q = part[k];
                              if (q.bad || T + q.mn < LO1 || T + q.mx > HI1) break;
                              T += q.tot;
                        }
                        s2 = __dmul_rn(__ll2double_rn(T), b.u);
                        p2 = pos + (long)k * RUN_W;
                        if (k < RUN_NW && p2 < n) {  // window k walked term by term
                              const int wk = n - p2 < RUN_W ? (int)(n - p2) : RUN_W;
                              s2 = run_window(stage + k * 32 * RUN_ROW, 0, wk, s2);
                              p2 += wk;
                        }
                  } else {
                        s2 = run_window(stage, 0, wl, s);  // this warp's window 0
                        p2 = pos + wl;
                  }
                  if (lane == 0) {
                        sh_s = s2;
                        sh_pos = p2 < n ? p2 : n;
                  }
            }
            __syncthreads();
            s = sh_s;
            pos = sh_pos;
            __syncthreads();
      }
      return s;
}

// Device error word bits (set by kernels instead of trapping).
enum : unsigned {
      ERR_CAPACITY = 1u,
      ERR_NMAX = 2u,
      ERR_TIMEOUT = 4u,
      ERR_INTERNAL = 8u,
      ERR_FRAGMENT = 16u,
};

// Scratch and state owned by the library, sized from n_max at ncgpu_init.
struct Ctx {
      int inited = 0;
      int n_max = 0;
      int sm_count = 148;      // multiprocessors of the current device (set by ncgpu_init)
      int grav_slots_mult = 32; // tiled gravity: CTAs per resident CTA slot (measured best of 2..32)
      ncgpu_params P{};
      cudaStream_t s = nullptr;

      // device-resident body state (SoA, FP64) + exists flags
      double *x = nullptr, *y = nullptr, *z = nullptr;
      double *vx = nullptr, *vy = nullptr, *vz = nullptr;
      double *m = nullptr, *R = nullptr;
      int *ex = nullptr;
      int *exs = nullptr;          // scratch exists flags for stateless calls
      int largest_id = -1;
      int uploaded = 0;
      double *cm = nullptr;        // 16 doubles: central mass record (8), SideralOmega at [8]
      double j2 = 0.;              // the J2 in force for the state's kicks (set at upload and end of step)
      double j2_prev = 0.;         // the J2 in force before the last end of step's update
      int com_reduced = 0;         // the last end of step reduced the barycentre
      int eot_lid = -1;            // largest_id at the start of the last end of step
      // output staging (output.cu): snapshot body fields and central body, the
      // formatter's slots / packed text / lengths
      double *snap[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
      double *snap_cm = nullptr;
      int snap_active = 0;
      char *fmt_slots = nullptr, *fmt_text = nullptr;
      int *fmt_len = nullptr;
      size_t fmt_cap = 0;
      // elliptic output (output.cu): per existing body a, lambda, k, h, q, p
      // (6 blocks), the atan2 arguments (2), the caller's atan2 (1), the caller's
      // elements of the bodies it converts itself (6 a body), a branch code
      // a body and the list of those bodies
      double *ell = nullptr;
      size_t ell_cap = 0;          // bodies
      unsigned char *ell_code = nullptr;
      int *ell_list = nullptr;     // [0]: count, then compact indices
      int ell_n = -1;              // bodies of the pending elliptic output (-1: none)
      int ell_nhost = 0;
      int ell_done = 0;            // lambda finished from the caller's atan2
      double *cm_acc = nullptr;    // 3 doubles
      double dt = 0.0;

      // gravity scratch
      double *acc = nullptr;       // 3 * n_max (x block, y block, z block)
      double *cmterm = nullptr;    // 6 * n_max (CM_acc terms; two per body with J2)
      double *partial = nullptr;   // gravity partial sums (chunks x 3 x n_max)
      size_t partial_cap = 0;      // doubles
      int *cidx = nullptr;         // compacted existing slot ids
      int *cnt = nullptr;          // block counts for compaction/scans
      int *n_dev = nullptr;        // small device scalars
      void *src64 = nullptr;       // packed FP64 sources (double4 per body)
      double *srcR = nullptr;      // softening * R per body (FP64)
      void *src32 = nullptr;       // packed FP32 sources (float4 per body)
      float *srcR32 = nullptr;
      double *tilebox = nullptr;   // per tile: cx,cy,cz,hx,hy,hz (6 doubles)
      uint32_t *keys = nullptr, *keys2 = nullptr;
      int *vals = nullptr, *vals2 = nullptr;
      int *hist = nullptr;         // radix histogram scratch
      size_t hist_cap = 0;
      double *red = nullptr;       // reduction scratch (bbox etc.)
      unsigned *err = nullptr;     // device error word
      double *aos = nullptr;       // 8 * n_max staging for host AoS copies
      double *pinned = nullptr;    // pinned host staging (8 * n_max doubles)
      cudaEvent_t kev0 = nullptr, kev1 = nullptr;  // bracket the dominant kernel
      int kev_valid = 0;
      // display()'s statistics, started by ncgpu_format_cartesian on a second
      // stream while its text crosses to the host; ncgpu_output_stats takes
      // them when no other entry point ran in between (any other one first
      // makes the main stream wait for them and drops them)
      cudaStream_t s2 = nullptr;
      cudaEvent_t sev0 = nullptr, sev1 = nullptr;
      // the output text's copies to the host, chunk by chunk behind the formatting
      cudaStream_t s3 = nullptr;
      cudaEvent_t cev = nullptr;
      int stats_pre = 0;

      // collision state (device)
      int *did = nullptr;          // did_collide[] (src/structure.c)
      unsigned char *dirty = nullptr;  // bodies modified by an event of the current sweep
      int *dlist = nullptr;        // their ids, in event order
      int *free_idx = nullptr;     // free_indexes[] stack (src/structure.c:849-878)
      int *scal = nullptr;         // device scalars, see enum Scal
      int *hi = nullptr, *hj = nullptr;   // candidate hits (i, j) of a sweep
      int hit_cap = 0;
      int *ev = nullptr;           // events: (a, b, type) per collision_treatment call
      double *evrec = nullptr;     // per-event record for the collision output file
      int ev_cap = 0;
      int n_events = 0;            // events of the last sweep (host copy)
      int collision_count = 0;     // collision_count (host copy)

      // mesh search (allocated on the first mesh pass)
      int2 *crange = nullptr;      // dense cell -> [first, end) of its bodies in the sorted keys ({-1, -1} empty)
      size_t cell_cap = 0;
      int mesh_d = 0;
      uint32_t *mkeys = nullptr;   // cell index per sorted body (n + 1, sentinel)
      int *mvals = nullptr;        // body index per sorted position
      int *mpv = nullptr;          // per sorted position: the body index if it exists, else INT_MAX
      double *gpart = nullptr;     // mesh gravity: per sorted position x, y, z, partner mass (4 doubles)
      // a mesh pass whose counts come back with the end of step's read (its
      // candidates' total, the small bodies' total before the drops)
      int mesh_pending = 0;
      long mesh_base = 0, mesh_small_total = 0;
      double *lf_buf = nullptr;    // the differentiable leapfrog's buffers (kept between calls)
      size_t lf_cap = 0;           // doubles
      int *ckey = nullptr;         // insertion cell per slot (-1: not inserted)
      int *mcnt = nullptr, *moff = nullptr;
      int *cand_k = nullptr, *cand_p = nullptr;  // candidates in pop order
      unsigned char *cflag = nullptr;
      int *cpos = nullptr;         // output positions of kept candidates
      int *msums = nullptr;        // scan scratch for candidate-sized scans
      long pair_cap = 0;
      int *occ = nullptr;
      void *mrec = nullptr;        // cell-ordered body records of a mesh pass (64 B each, n_max)
      int occ_cap = 0;
      // fragmentation in a mesh pass: per-event records (EVX ints: candidate
      // position, extra-pair offset, extra-pair count, first tail fragment,
      // largest fragment A, next full fragmentation of the same A), the tail's
      // pairs, per-slot heads of those chains (-1), full events in order
      int *evx = nullptr;
      int *xpairs = nullptr;
      long xpair_cap = 0;
      int *xhead = nullptr;
      int *fev = nullptr;
      int mesh_nev = 0;            // events recorded by the last mesh pass
      int mesh_nfev = 0;           // full fragmentations of the last mesh pass
      int mesh_nx = 0;             // extra pairs of the last mesh pass
      // visits of bodies larger than the mesh size in the last mesh pass:
      // (body, first candidate, end) in visit order
      int *vis = nullptr;
      int vis_host[3 * 1024];
      int mesh_nvis = 0;
      int mesh_valid = 0;          // cell table populated by the last pass
      int mesh_n = 0;              // sorted entries of the last pass (largest_id + 1)
      int n_cand = 0, n_pairs = 0;
      long total_neighbours = 0;
      int how_many_small = 0, how_many_big = 0;
      int force_naive = 0;         // force_naive_bool: brute force below switch_to_brute_force
};

// Indices into Ctx::scal (device ints).
enum Scal : int {
      S_LID = 0,        // largest_id
      S_NFREE = 1,      // how_many_free
      S_NHITS = 2,      // hits appended by a sweep
      S_NEV = 3,        // events of the current sweep
      S_NDIRTY = 4,     // entries in dlist
      S_CCOUNT = 5,     // collision_count
      S_NPAIRS = 6,     // pairs appended (mesh)
      S_HM = 7,         // how_many_moonlets
      S_NFLAG = 8,      // bodies flagged for dumping
      S_NEEDCOM = 9,    // need_to_reduce_COM_bool
      S_NBIG = 10,      // bodies larger than the mesh size
      S_NDROP = 11,     // candidates dropped by removals
      S_NINS = 12,      // bodies inserted in the cell table
      S_FMERGE = 13,    // merger_count (fragmentation model outcomes, src/structure.h:148-151)
      S_FSUPER = 14,    // super_catastrophic_count
      S_FHALF = 15,     // half_fragmentation_count
      S_FFULL = 16,     // full_fragmentation_count
      S_NXPAIRS = 17,   // fragment pairs appended by a mesh pass (extra pairs)
      S_NSKIP = 18,     // mesh event candidates that append no pair of their own
      S_NFEV = 19,      // full fragmentations of a mesh pass
      S_COUNT = 24
};

// Per-event record fields (doubles) kept for the collision output file
// (collisionData, src/display.c): t_coll, m_A, m_B, R_A, R_B, DeltaV, dr.dv.
constexpr int EVREC = 8;
// Per-event ints of a mesh pass (see Ctx::evx).
constexpr int EVX = 8;
// Visits of bodies larger than the mesh size recorded per mesh pass.
constexpr int MAX_VISITS = 1024;

Ctx &ctx();
int ensure_partial(size_t doubles);
int check_err_word();        // syncs the stream, reads and clears the device error word
int sync_scalars_h(int *h);  // device scalars into c.* and h[S_COUNT], error word checked (one sync)

// Gravity driver (gravity.cu).  Reads bodies through `bv` for slots
// 0..largest_id, writes acc (3 blocks of n_max: ax, ay, az, zero for empty
// slots) and cm_acc (3 doubles, device).
// With nparts > 1 only the targets of part `part` get their acceleration (the
// compacted order's part-th slice in the exact mode, the part-th slice of the
// Morton-ordered target blocks in the tiled modes); every other row gets -0.0
// (+0.0 for empty slots from part 0), so that the sum over the parts is the
// full field, bit for bit.  CM_acc is the full one in every part.
// cm_dev (may be null): the central body in device memory; the exact mode up to
// EXACT_SMALL_N body slots then runs without reading anything back.
constexpr int EXACT_SMALL_N = 8192;
int gravity_eval(const BodyView &bv, int largest_id, const double *cm_host8, const J2Arg &j2, double *d_acc,
                 long acc_stride_block, double *d_cm_acc, int mode, cudaStream_t st, int part = 0, int nparts = 1,
                 const double *cm_dev = nullptr);

// Sequential FP64 sums, in index order, of the 3 arrays terms[c*n .. c*n + n),
// starting from init[c] (0 when init is null); out may alias init.
int seq_sum3(const double *terms, int n, const double *init, double *out, cudaStream_t st);
// The same sums as a deterministic two-level parallel reduction (non-exact
// gravity modes), added to init[c] at the end.
int par_sum3(const double *terms, int n, const double *init, double *out, cudaStream_t st);

// tides (src/physics.c:496-542) on the device state after the vector field
// (tides.cu): acc blocks of n_max and the device CM_acc receive the tidal
// terms, SideralOmega (cm[8]) changes body by body.
int tides_state(double *d_acc, long acc_stride_block, double *d_cm_acc);

// The central mass record and SideralOmega of the device state (9 doubles).
int state_cm_host(double *cm9);

// Re-evaluates the J2 in force (ctx().j2) from the device state.
int refresh_j2();

// LSD radix sort of (key, value) pairs, stable; keys use `bits` low bits.
// Result ends in (keys, vals) buffers passed in (ping-pong through ctx scratch).
int radix_sort_pairs(uint32_t *keys, int *vals, int n, int bits, cudaStream_t st);

// Exclusive prefix sum; out has n + 1 entries (out[n] = total).
int scan_exclusive(const int *in, int *out, int n, int *sums, cudaStream_t st);

// Stream compaction of existing slots 0..largest_id into ctx().cidx (ascending).
// Returns the count through *n_host (synchronises).
int compact_existing(const int *ex, int largest_id, int *n_host, cudaStream_t st);
// The same compaction without the synchronisation: the count stays in
// ctx().n_dev[0].
int compact_existing_dev(const int *ex, int largest_id, cudaStream_t st);

// Compaction of flagged slots with caller-provided scratch (no library context).
int compact_flags_into(const int *flags, int n_slots, int *blockcnt, int *n_dev, int *out_idx, int *n_host,
                       cudaStream_t st);

// The exact gravity on caller-provided scratch (no library context).
int gravity_exact_into(const BodyView &bv, int largest_id, const double *cmh, double G, double sp, int central,
                       const J2Arg &j2, int *cidx, double *src, double *srcR, double *cterm, int *blockcnt,
                       int *n_dev, unsigned *err, double *ax, double *ay, double *az, double *d_cm_acc,
                       cudaStream_t st);

}  // namespace ncg
