// Output staging on the device: the text display() writes at an output step
// (src/display.c:239-451) for the cartesian files, and the statistics of its
// stat.txt line, computed from the device state.
//
// Snapshot.  At an output step the drivers apply a half backward drift (brute
// force, src/rk4.c:881-890) or a half backward kick (mesh, src/rk4.c:740-757) to
// a copy of the bodies, print the copy and go on with the original.  The copy
// shares the reference's globals with the original: exists[], the free-index
// stack, largest_id and SideralOmega.  ncgpu_snapshot_begin copies the body
// fields and the central body into snapshot arrays and makes them the state
// (every entry point then works on the copy, with exists[] and the free slots
// shared); ncgpu_snapshot_end makes the original the state again and carries
// the copy's SideralOmega over (the tides of the backward kick change it).
// Between the two calls every entry point works on the copy.
//
// Formatting.  "%.14lf " of a double is the decimal of its exact binary value
// rounded to 14 fractional digits, ties to even (glibc's printf).  With
// x = m 2^e (m < 2^53), |x| 10^14 = m 5^14 2^(e+14): the product m 5^14 < 2^86
// fits a 128-bit integer, the power of two is a shift, and the rounding of a
// right shift is exact integer arithmetic.  Values whose |x| 10^14 reaches 2^127
// (|x| > 1.7e24) are not formatted (NCGPU_E_UNSUPPORTED; the caller prints them).
#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

#include "common.cuh"
#include "physics.cuh"

namespace ncg {

int compact_existing(const int *ex, int largest_id, int *n_host, cudaStream_t st);

namespace {

constexpr int SLOT = 48;  // bytes per formatted value (at most 42 used)

// "%.14lf " of v into out (at most 42 bytes); returns the length, or -1 when
// |v| 10^14 does not fit 127 bits.
__device__ int fmt_fixed14(double v, char *out)
{
      const unsigned long long bits = (unsigned long long)__double_as_longlong(v);
      const bool neg = bits >> 63;
      const int be = (int)((bits >> 52) & 0x7ff);
      const unsigned long long frac = bits & 0xfffffffffffffull;
      int k = 0;
      if (be == 0x7ff) {  // inf / nan, as glibc prints them with %lf
            if (neg) out[k++] = '-';
            const char *w = frac ? "nan" : "inf";
            for (int i = 0; i < 3; i++) out[k++] = w[i];
            out[k++] = ' ';
            return k;
      }
      const unsigned long long m = be ? (frac | (1ull << 52)) : frac;
      const int e = be ? be - 1075 : -1074;  // v = +-m 2^e
      constexpr unsigned long long P5_14 = 6103515625ull;  // 5^14
      unsigned __int128 P = (unsigned __int128)m * P5_14;
      const int s = e + 14;
      unsigned __int128 N;
      if (s >= 0) {
            if (P != 0 && (s >= 127 || (P >> (127 - s)) != 0)) return -1;
            N = P << s;
      } else {
            const int r = -s;
            if (r >= 128) {
                  N = 0;  // P < 2^86 < half of 2^r
            } else {
                  const unsigned __int128 q = P >> r;
                  const unsigned __int128 rem = P - (q << r);
                  const unsigned __int128 half = (unsigned __int128)1 << (r - 1);
                  N = (rem > half || (rem == half && (q & 1))) ? q + 1 : q;
            }
      }
      if (neg) out[k++] = '-';
      const unsigned __int128 TEN14 = (unsigned __int128)100000000000000ull;
      unsigned __int128 ip = N / TEN14;
      unsigned long long fp = (unsigned long long)(N - ip * TEN14);
      char d[40];
      int nd = 0;
      do {
            d[nd++] = (char)('0' + (int)(ip % 10));
            ip /= 10;
      } while (ip != 0);
      while (nd > 0) out[k++] = d[--nd];
      out[k++] = '.';
      for (int i = 13; i >= 0; --i) {
            out[k + i] = (char)('0' + (int)(fp % 10));
            fp /= 10;
      }
      k += 14;
      out[k++] = ' ';
      return k;
}

// The values of the cartesian files, value i of the concatenation: files 0..5
// (x y z vx vy vz, the central body first when `central`), then 6, 7 (mass and
// radius of the bodies only).
struct CartValues {
      BodyView S;
      const double *cm;
      const int *cidx;
      int n, central;
      __device__ __forceinline__ double operator()(long i) const
      {
            const int per = n + central;
            int f, j;
            if (i < 6L * per) {
                  f = (int)(i / per);
                  j = (int)(i % per);
            } else {
                  f = 6 + (int)((i - 6L * per) / n);
                  j = (int)((i - 6L * per) % n);
            }
            const int c = f < 6 ? central : 0;
            if (j < c) return cm[f];
            const long s = (long)cidx[j - c] * S.stride;
            const double *a[8] = {S.x, S.y, S.z, S.vx, S.vy, S.vz, S.m, S.R};
            return a[f][s];
      }
};

// The values of the elliptic files: a, lambda, k, h, q, p of the bodies (six
// blocks of n), then their masses and radii.
struct EllValues {
      BodyView S;
      const double *ell;  // six blocks, `stride` doubles apart
      const int *cidx;
      int n;
      long stride;
      __device__ __forceinline__ double operator()(long i) const
      {
            const int f = (int)(i / n), j = (int)(i % n);
            if (f < 6) return ell[f * stride + j];
            return (f == 6 ? S.m : S.R)[(long)cidx[j] * S.stride];
      }
};

// One thread per value: formatted into its slot, the length into len.
template <class Values>
__global__ void k_fmt_values(Values val, long lo, long hi, char *__restrict__ slots, int *__restrict__ len,
                             unsigned *err)
{
      const long i = lo + (long)blockIdx.x * blockDim.x + threadIdx.x;
      if (i >= hi) return;
      const int L = fmt_fixed14(val(i), slots + (size_t)i * SLOT);
      if (L < 0) atomicOr(err, ERR_INTERNAL);
      len[i] = L < 0 ? 0 : L;
}

// Copies the slots of values lo .. hi-1 to their places in the packed text
// (offsets: exclusive scan of those values' lengths, from text; the files'
// texts follow one another, without newlines).
__global__ void k_fmt_pack(const char *__restrict__ slots, const int *__restrict__ off, long lo, long hi,
                           char *__restrict__ text)
{
      const long i = lo + (long)blockIdx.x * blockDim.x + threadIdx.x;
      if (i >= hi) return;
      const int L = off[i + 1] - off[i];
      const char *src = slots + (size_t)i * SLOT;
      char *dst = text + off[i];
      for (int c = 0; c < L; c++) dst[c] = src[c];
}

// display()'s statistics of the bodies (src/display.c:303-379): the total mass,
// summed in slot order, and the two most massive bodies as its loop picks them
// (strictly greater replaces, so the first of equal masses wins; i1 = i2 = 0 and
// M = 0 when there are fewer positive masses).
// The two most massive bodies (src/display.c:353-363): the reference scans the
// slots in ascending order from M = 0 with strict comparisons, which keeps the
// first two positive masses of the order (mass descending, slot ascending).
// That order is total, so the scan is a reduction: each thread keeps the first
// two of its bodies, then threads, warps and blocks merge their pairs.
struct Top2 {
      double M1, M2;
      int i1, i2;
};

__device__ __forceinline__ bool top_before(double a, int i, double b, int j) { return a > b || (a == b && i < j); }

__device__ __forceinline__ void top2_insert(Top2 &t, double m, int p)
{
      if (top_before(m, p, t.M1, t.i1)) {
            t.M2 = t.M1;
            t.i2 = t.i1;
            t.M1 = m;
            t.i1 = p;
      } else if (top_before(m, p, t.M2, t.i2)) {
            t.M2 = m;
            t.i2 = p;
      }
}

__device__ __forceinline__ void top2_warp(Top2 &t)
{
      for (int o = 16; o > 0; o >>= 1) {
            const double b1 = __shfl_xor_sync(0xffffffffu, t.M1, o), b2 = __shfl_xor_sync(0xffffffffu, t.M2, o);
            const int k1 = __shfl_xor_sync(0xffffffffu, t.i1, o), k2 = __shfl_xor_sync(0xffffffffu, t.i2, o);
            top2_insert(t, b1, k1);
            top2_insert(t, b2, k2);
      }
}

constexpr int TOP_T = 256, TOP_MAXB = 148 * 8;

// The compacted masses m[q] = S.m[cidx[q]] (the sequential total's input) and
// each block's first two bodies: pm[2b], pm[2b+1] with slots pi[2b], pi[2b+1]
// (mass 0 and slot INT_MAX for an empty entry).
__global__ void __launch_bounds__(TOP_T) k_out_top2(BodyView S, const int *__restrict__ cidx, int n,
                                                    double *__restrict__ m, double *__restrict__ pm,
                                                    int *__restrict__ pi)
{
      __shared__ Top2 wt[TOP_T / 32];
      Top2 t{0., 0., 0x7fffffff, 0x7fffffff};
      for (int q = blockIdx.x * TOP_T + threadIdx.x; q < n; q += gridDim.x * TOP_T) {
            const int p = cidx[q];
            const double v = S.m[(long)p * S.stride];
            m[q] = v;
            if (v > 0.) top2_insert(t, v, p);
      }
      top2_warp(t);
      const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
      if (lane == 0) wt[w] = t;
      __syncthreads();
      if (w == 0) {
            t = lane < TOP_T / 32 ? wt[lane] : Top2{0., 0., 0x7fffffff, 0x7fffffff};
            top2_warp(t);
            if (lane == 0) {
                  pm[2 * blockIdx.x] = t.M1;
                  pm[2 * blockIdx.x + 1] = t.M2;
                  pi[2 * blockIdx.x] = t.i1;
                  pi[2 * blockIdx.x + 1] = t.i2;
            }
      }
}

__global__ void k_gather_mass(BodyView S, const int *__restrict__ cidx, int n, double *__restrict__ m)
{
      const int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q < n) m[q] = S.m[(long)cidx[q] * S.stride];
}

__global__ void k_gather_radius(BodyView S, const int *__restrict__ cidx, int n, double *__restrict__ r)
{
      const int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q < n) r[q] = S.R[(long)cidx[q] * S.stride];
}

// The blocks' pairs merged (out[1], out[2]; the slots in out_idx, 0 when a
// mass is absent, as the reference leaves them), then the total mass out[0]:
// the masses summed in slot order with round-to-nearest, the reference's sum
// (taken in runs from RUN_SUM_MIN bodies on).
constexpr int RUN_SUM_MIN = 65536;
__global__ void __launch_bounds__(RUN_NW * 32) k_chain_total(const double *__restrict__ m, int n,
                                                             double *__restrict__ out, const double *__restrict__ pm,
                                                             const int *__restrict__ pi, int nb,
                                                             int *__restrict__ out_idx)
{
      extern __shared__ __align__(16) double stage[];  // RUN_STAGE doubles
      if (threadIdx.x < 32) {
            Top2 t{0., 0., 0x7fffffff, 0x7fffffff};
            for (int k = threadIdx.x; k < 2 * nb; k += 32) top2_insert(t, pm[k], pi[k]);
            top2_warp(t);
            if (threadIdx.x == 0) {
                  out[1] = t.M1;
                  out[2] = t.M2;
                  out_idx[0] = t.M1 > 0. ? t.i1 : 0;
                  out_idx[1] = t.M2 > 0. ? t.i2 : 0;
            }
      }
      if (n >= RUN_SUM_MIN) {
            const double s = block_run_sum(m, n, 0., stage);
            if (threadIdx.x == 0) out[0] = s;
      } else if (threadIdx.x < 32) {
            const double s = warp_chain_sum(m, n, 0., stage);
            if (threadIdx.x == 0) out[0] = s;
      }
}

// ---- elliptic elements (cart2ell, src/structure.c:172-284) ----------------

enum { ELL_ATAN2 = 0, ELL_ZERO = 1, ELL_HOST = 2 };

// cart2ell of one body up to its mean longitude's atan2, in the reference's
// operation order with round-to-nearest FP64 intrinsics (no FMA
// contraction), so that a, k, h, q, p and the atan2 arguments are the
// reference's bit for bit.  code:
//   ELL_ATAN2  the elliptic branch: lambda = atan2(sinF, cosF) - l, the atan2
//              left to the caller's libm (the function the reference calls);
//   ELL_ZERO   R or V2 zero: lambda = 0 (src/structure.c:262-264);
//   ELL_HOST   the caller converts the body with the reference's cart2ell: the
//              hyperbolic branch (atanh, sinh; src/structure.c:274-279), the
//              (k, h) warning the reference prints (src/structure.c:253-255),
//              or a NaN anywhere (the device's NaNs do not carry the host's
//              signs, which printf shows).
struct Ell {
      double a, l, k, h, q, p, sinF, cosF;
      int code;
};

__device__ Ell d_cart2ell(double X, double Y, double Z, double vX, double vY, double vZ, const double *cmb,
                          bool central, bool j2, double J2, double R_unit, double mu)
{
      Ell e;
      e.l = e.sinF = e.cosF = 0.;
      e.code = ELL_ATAN2;
      X = DSUB(X, central ? cmb[0] : 0.);
      Y = DSUB(Y, central ? cmb[1] : 0.);
      Z = DSUB(Z, central ? cmb[2] : 0.);
      vX = DSUB(vX, central ? cmb[3] : 0.);
      vY = DSUB(vY, central ? cmb[4] : 0.);
      vZ = DSUB(vZ, central ? cmb[5] : 0.);
      // semi-major axis, with the J2 correction of Kepler's third law
      const double R = __dsqrt_rn(DADD(DADD(DMUL(X, X), DMUL(Y, Y)), DMUL(Z, Z)));
      double V2 = DADD(DADD(DMUL(vX, vX), DMUL(vY, vY)), DMUL(vZ, vZ));
      double AA = DDIV(DMUL(R, mu), DSUB(DMUL(2., mu), DMUL(R, V2)));
      if (j2 && AA > 0.) {
            mu = DMUL(mu, DADD(1., DDIV(DMUL(DMUL(DMUL(1., J2), R_unit), R_unit), DMUL(AA, AA))));
            AA = DDIV(DMUL(R, mu), DSUB(DMUL(2., mu), DMUL(R, V2)));
      }
      e.a = AA;
      // velocities in units of sqrt(mu), angular momentum
      const double SMU = __dsqrt_rn(mu);
      vX = DDIV(vX, SMU);
      vY = DDIV(vY, SMU);
      vZ = DDIV(vZ, SMU);
      V2 = DADD(DADD(DMUL(vX, vX), DMUL(vY, vY)), DMUL(vZ, vZ));
      const double RV = DADD(DADD(DMUL(X, vX), DMUL(Y, vY)), DMUL(Z, vZ));
      const double C1 = DSUB(DMUL(Y, vZ), DMUL(Z, vY));
      const double C2 = DSUB(DMUL(Z, vX), DMUL(X, vZ));
      const double C3 = DSUB(DMUL(X, vY), DMUL(Y, vX));
      const double CC = DADD(DADD(DMUL(C1, C1), DMUL(C2, C2)), DMUL(C3, C3));
      const double DC = __dsqrt_rn(CC);
      // (q, p)
      const double aux0 = __dsqrt_rn(DMUL(2., DADD(CC, DMUL(DC, C3))));
      e.q = aux0 == 0. ? 0. : DDIV(-C2, aux0);
      e.p = aux0 == 0. ? 0. : DDIV(C1, aux0);
      if (R == 0. || V2 == 0.) {
            e.k = e.h = 0.;
            e.code = ELL_ZERO;
      } else {
            // (k, h)
            const double a11 = DSUB(V2, DDIV(1., R));
            const double a12 = DDIV(RV, DMUL(R, DC));
            const double a21 = -RV;
            const double a22 = DSUB(DC, DDIV(R, DC));
            const double c11 = DADD(DMUL(X, a11), DMUL(vX, a21));
            const double c12 = DADD(DMUL(X, a12), DMUL(vX, a22));
            const double c21 = DADD(DMUL(Y, a11), DMUL(vY, a21));
            const double c22 = DADD(DMUL(Y, a12), DMUL(vY, a22));
            const double FAC1 = DDIV(C1, DADD(DC, C3));
            const double FAC2 = DDIV(C2, DADD(DC, C3));
            const double K1 = DSUB(c11, DMUL(FAC1, DADD(DMUL(Z, a11), DMUL(vZ, a21))));
            const double H1 = DADD(-c12, DMUL(FAC1, DADD(DMUL(Z, a12), DMUL(vZ, a22))));
            const double H2 = DSUB(c21, DMUL(FAC2, DADD(DMUL(Z, a11), DMUL(vZ, a21))));
            const double K2 = DSUB(c22, DMUL(FAC2, DADD(DMUL(Z, a12), DMUL(vZ, a22))));
            const bool warn = DADD(fabs(DSUB(H1, H2)), fabs(DSUB(K1, K2))) > 1.e-6;
            e.k = DMUL(0.5, DADD(K1, K2));
            e.h = DMUL(0.5, DADD(H1, H2));
            // mean longitude, elliptic branch (sqrt of a negative is NaN: hyperbolic)
            const double USQA = __dsqrt_rn(DSUB(DDIV(2., R), V2));
            if (USQA >= 0. && !warn) {
                  const double b12 = DSUB(vX, DMUL(FAC1, vZ));
                  const double b22 = DSUB(vY, DMUL(FAC2, vZ));
                  const double aux1 = DDIV(DSUB(DMUL(R, V2), 1.), DADD(1., DMUL(DC, USQA)));
                  e.sinF = DADD(DMUL(DMUL(-b12, R), USQA), DMUL(e.h, aux1));
                  e.cosF = DADD(DMUL(DMUL(b22, R), USQA), DMUL(e.k, aux1));
                  e.l = DMUL(RV, USQA);
            } else {
                  e.code = ELL_HOST;
            }
      }
      if (isnan(e.a) || isnan(e.k) || isnan(e.h) || isnan(e.q) || isnan(e.p) || isnan(e.l) || isnan(e.sinF) ||
          isnan(e.cosF))
            e.code = ELL_HOST;
      return e;
}

// One thread per existing body j (slot cidx[j]), with display()'s
// mu + G m (src/display.c:341).  Writes the six element blocks, N doubles
// apart (lambda's block holds l until k_ell_lambda), the atan2 arguments
// (y, x) and the branch code,
// and lists the ELL_HOST bodies (list[0]: their count).
__global__ void k_cart2ell(BodyView S, const double *__restrict__ cmb, const int *__restrict__ cidx, int n,
                           double mu, double G, int central, int j2, double J2, double R_unit,
                           double *__restrict__ ell, long N, double *__restrict__ yx,
                           unsigned char *__restrict__ code, int *__restrict__ list)
{
      const int j = blockIdx.x * blockDim.x + threadIdx.x;
      if (j >= n) return;
      const long s = (long)cidx[j] * S.stride;
      const Ell e = d_cart2ell(S.x[s], S.y[s], S.z[s], S.vx[s], S.vy[s], S.vz[s], cmb, central != 0, j2 != 0, J2,
                               R_unit, DADD(mu, DMUL(G, S.m[s])));
      ell[j] = e.a;
      ell[N + j] = e.l;
      ell[2 * N + j] = e.k;
      ell[3 * N + j] = e.h;
      ell[4 * N + j] = e.q;
      ell[5 * N + j] = e.p;
      yx[2 * (long)j] = e.sinF;
      yx[2 * (long)j + 1] = e.cosF;
      code[j] = (unsigned char)e.code;
      if (e.code == ELL_HOST) list[1 + atomicAdd(list, 1)] = j;
}

// The records and slots of the listed bodies, for the caller's cart2ell.
__global__ void k_ell_gather(BodyView S, const int *__restrict__ cidx, const int *__restrict__ list, int nh,
                             double *__restrict__ rec, int *__restrict__ slot)
{
      const int k = blockIdx.x * blockDim.x + threadIdx.x;
      if (k >= nh) return;
      const int b = cidx[list[k]];
      const long s = (long)b * S.stride;
      double *r = rec + 8 * (long)k;
      r[0] = S.x[s]; r[1] = S.y[s]; r[2] = S.z[s]; r[3] = S.vx[s]; r[4] = S.vy[s]; r[5] = S.vz[s];
      r[6] = S.m[s]; r[7] = S.R[s];
      slot[k] = b;
}

// lambda = F - RV USQA (src/structure.c:272) from the caller's F = atan2(sinF, cosF).
__global__ void k_ell_lambda(const double *__restrict__ F, const unsigned char *__restrict__ code,
                             double *__restrict__ lam, int n)
{
      const int j = blockIdx.x * blockDim.x + threadIdx.x;
      if (j < n && code[j] == ELL_ATAN2) lam[j] = DSUB(F[j], lam[j]);
}

// The caller's elements of the listed bodies (six a body, alkhqp order) into
// the element blocks, `stride` doubles apart.
__global__ void k_ell_host(const int *__restrict__ list, const double *__restrict__ alk, int nh,
                           double *__restrict__ ell, long stride)
{
      const int k = blockIdx.x * blockDim.x + threadIdx.x;
      if (k >= nh) return;
      const long j = list[k];
      for (int f = 0; f < 6; f++) ell[f * stride + j] = alk[6 * (long)k + f];
}

}  // namespace
}  // namespace ncg

using namespace ncg;

namespace ncg {
BodyView state_view();
int scan_exclusive(const int *in, int *out, int n, int *sums, cudaStream_t st);
}

extern "C" int ncgpu_snapshot_begin(void)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      if (c.snap_active) return NCGPU_E_STATE;
      const size_t N = (size_t)c.n_max;
      if (!c.snap[0]) {
            for (int f = 0; f < 8; f++) NCG_CK(cudaMalloc(&c.snap[f], N * sizeof(double)));
            NCG_CK(cudaMalloc(&c.snap_cm, 16 * sizeof(double)));
      }
      double **fld[8] = {&c.x, &c.y, &c.z, &c.vx, &c.vy, &c.vz, &c.m, &c.R};
      const size_t ns = (size_t)(c.largest_id + 1);
      for (int f = 0; f < 8; f++) {
            if (ns > 0) NCG_CK(cudaMemcpyAsync(c.snap[f], *fld[f], ns * sizeof(double), cudaMemcpyDeviceToDevice, c.s));
            double *t = *fld[f];
            *fld[f] = c.snap[f];
            c.snap[f] = t;
      }
      NCG_CK(cudaMemcpyAsync(c.snap_cm, c.cm, 16 * sizeof(double), cudaMemcpyDeviceToDevice, c.s));
      double *t = c.cm;
      c.cm = c.snap_cm;
      c.snap_cm = t;
      c.snap_active = 1;
      return NCGPU_OK;
}

extern "C" int ncgpu_snapshot_end(void)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.snap_active) return NCGPU_E_STATE;
      double **fld[8] = {&c.x, &c.y, &c.z, &c.vx, &c.vy, &c.vz, &c.m, &c.R};
      for (int f = 0; f < 8; f++) {
            double *t = *fld[f];
            *fld[f] = c.snap[f];
            c.snap[f] = t;
      }
      // SideralOmega is one global in the reference: the copy's value stays
      NCG_CK(cudaMemcpyAsync(c.snap_cm + 8, c.cm + 8, sizeof(double), cudaMemcpyDeviceToDevice, c.s));
      double *t = c.cm;
      c.cm = c.snap_cm;
      c.snap_cm = t;
      c.snap_active = 0;
      NCG_CK(cudaStreamSynchronize(c.s));
      return NCGPU_OK;
}

extern "C" unsigned long ncgpu_format_cartesian_cap(void)
{
      Ctx &c = ctx();
      if (!c.inited) return 0;
      return 8ul * ((unsigned long)c.n_max + 1ul) * 42ul;
}

namespace ncg {
namespace {

// Formats `total` values (file f: values first[f] .. first[f + 1] - 1) and
// copies the files' texts, one after the other, into text; lens[f] receives
// each file's length.  In chunks of FMT_CHUNK values: a chunk's text crosses to
// the host on the copy stream while the next chunk is formatted.
// NCGPU_E_UNSUPPORTED when a value is beyond the formatter's range,
// NCGPU_E_CAPACITY when cap is too small (text then holds an unspecified
// prefix).
constexpr long FMT_CHUNK = 1L << 20;
template <class Values>
int format_files(const Values &val, int nfiles, const long *first, char *text, unsigned long cap, unsigned long *lens)
{
      Ctx &c = ctx();
      cudaStream_t st = c.s;
      const long total = first[nfiles];
      if (total >= 0x7fffffffL / SLOT) return NCGPU_E_CAPACITY;
      const size_t need = (size_t)(total > 0 ? total : 1) * SLOT;
      if (need > c.fmt_cap) {  // slots, packed text, lengths + offsets, scan sums
            if (c.fmt_slots) cudaFree(c.fmt_slots);
            if (c.fmt_text) cudaFree(c.fmt_text);
            if (c.fmt_len) cudaFree(c.fmt_len);
            c.fmt_slots = c.fmt_text = nullptr;
            c.fmt_len = nullptr;
            c.fmt_cap = 0;
            const size_t vals = need / SLOT;
            NCG_CK(cudaMalloc(&c.fmt_slots, need));
            NCG_CK(cudaMalloc(&c.fmt_text, need));
            NCG_CK(cudaMalloc(&c.fmt_len, sizeof(int) * (2 * vals + 2 + vals / 1024 + 2)));
            c.fmt_cap = need;
      }
      const size_t vals = c.fmt_cap / SLOT;
      int *len = c.fmt_len, *off = c.fmt_len + vals + 1, *sums = c.fmt_len + 2 * vals + 2;
      long h[16] = {0};
      int rel[17] = {0};  // [0..nfiles]: boundary offsets within their chunk; [16]: the chunk's length
      unsigned herr = 0;
      long base = 0;
      int st_ret = NCGPU_OK;
      for (long lo = 0; lo < total; lo += FMT_CHUNK) {
            const long hi = std::min(total, lo + FMT_CHUNK);
            const int nb = (int)((hi - lo + 255) / 256);
            k_fmt_values<<<nb, 256, 0, st>>>(val, lo, hi, c.fmt_slots, len, c.err);
            NCG_LAUNCHED();
            // chunk-relative offsets; off[hi] is the chunk's length until the next chunk's scan
            NCG_TRY(scan_exclusive(len + lo, off + lo, (int)(hi - lo), sums, st));
            k_fmt_pack<<<nb, 256, 0, st>>>(c.fmt_slots, off, lo, hi, c.fmt_text + base);
            NCG_LAUNCHED();
            for (int f = 0; f <= nfiles; f++)  // each boundary read with the chunk that starts at or holds it
                  if ((first[f] >= lo && first[f] < hi) || (first[f] == total && hi == total))
                        NCG_CK(cudaMemcpyAsync(&rel[f], off + first[f], sizeof(int), cudaMemcpyDeviceToHost, st));
            NCG_CK(cudaMemcpyAsync(&rel[16], off + hi, sizeof(int), cudaMemcpyDeviceToHost, st));
            NCG_CK(cudaMemcpyAsync(&herr, c.err, sizeof herr, cudaMemcpyDeviceToHost, st));
            NCG_CK(cudaStreamSynchronize(st));
            if (herr) break;
            for (int f = 0; f <= nfiles; f++)
                  if ((first[f] >= lo && first[f] < hi) || (first[f] == total && hi == total)) h[f] = base + rel[f];
            if ((unsigned long)(base + rel[16]) > cap) {
                  st_ret = NCGPU_E_CAPACITY;
                  break;
            }
            if (rel[16] > 0) {  // this chunk's text to the host, behind the previous chunks' copies
                  NCG_CK(cudaEventRecord(c.cev, st));
                  NCG_CK(cudaStreamWaitEvent(c.s3, c.cev, 0));
                  NCG_CK(cudaMemcpyAsync(text + base, c.fmt_text + base, (size_t)rel[16], cudaMemcpyDeviceToHost,
                                         c.s3));
            }
            base += rel[16];
      }
      NCG_CK(cudaStreamSynchronize(c.s3));
      if (total <= 0) {
            NCG_CK(cudaMemcpyAsync(&herr, c.err, sizeof herr, cudaMemcpyDeviceToHost, st));
            NCG_CK(cudaStreamSynchronize(st));
      }
      if (herr & ERR_INTERNAL) {  // a value beyond the formatter's range
            NCG_CK(cudaMemsetAsync(c.err, 0, sizeof(unsigned), st));
            return NCGPU_E_UNSUPPORTED;
      }
      if (herr) return check_err_word();
      if (st_ret != NCGPU_OK) return st_ret;
      for (int f = 0; f < nfiles; f++) lens[f] = (unsigned long)(h[f + 1] - h[f]);
      return NCGPU_OK;
}

}  // namespace
}  // namespace ncg

namespace ncg {
namespace {

// display()'s statistics of the n compacted bodies on stream st: the total mass
// and the two most massive bodies into c.red[3900..2], their slots into the
// two ints at c.red + 3904.
int stats_launch(int n, cudaStream_t st)
{
      Ctx &c = ctx();
      const size_t mcap = ((size_t)n + 8) & ~(size_t)7;
      NCG_TRY(ensure_partial(mcap + 3 * TOP_MAXB));
      double *m = c.partial, *pm = c.partial + mcap, *res = c.red + 3900;
      int *pi = (int *)(pm + 2 * TOP_MAXB), *didx = (int *)(c.red + 3904);
      const int nb = (int)std::min<long>(std::max<long>(((long)n + TOP_T - 1) / TOP_T, 1), TOP_MAXB);
      k_out_top2<<<nb, TOP_T, 0, st>>>(state_view(), c.cidx, n, m, pm, pi);
      NCG_LAUNCHED();
      constexpr int smem = RUN_STAGE * (int)sizeof(double);
      NCG_CK(cudaFuncSetAttribute(k_chain_total, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      k_chain_total<<<1, RUN_NW * 32, smem, st>>>(m, n, res, pm, pi, nb, didx);
      NCG_LAUNCHED();
      return NCGPU_OK;
}

}  // namespace
}  // namespace ncg

extern "C" int ncgpu_format_cartesian(char *text, unsigned long cap, unsigned long *lens)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      if (!text || !lens) return NCGPU_E_ARG;
      int n = 0;
      NCG_TRY(compact_existing(c.ex, c.largest_id, &n, c.s));
      // display()'s statistics on the second stream, while the text is formatted
      // and copied out; ncgpu_output_stats, called next, takes them
      NCG_CK(cudaEventRecord(c.sev0, c.s));
      NCG_CK(cudaStreamWaitEvent(c.s2, c.sev0, 0));
      NCG_TRY(stats_launch(n, c.s2));
      NCG_CK(cudaEventRecord(c.sev1, c.s2));
      c.stats_pre = 1;
      const int central = c.P.par_central_mass_bool ? 1 : 0;
      const long per = n + central;
      const long first[9] = {0, per, 2 * per, 3 * per, 4 * per, 5 * per, 6 * per, 6 * per + n, 6 * per + 2L * n};
      return format_files(CartValues{state_view(), c.cm, c.cidx, n, central}, 8, first, text, cap, lens);
}

namespace ncg {
namespace {

// The elliptic buffers for n bodies: ell (6n doubles: a, lambda, k, h, q, p),
// yx (2n: the atan2 arguments, then the caller's F), h (8n: the listed bodies'
// records, then the caller's elements), codes, the list (1 + n ints) and the
// listed bodies' slots (n ints).
int ensure_ell(size_t n)
{
      Ctx &c = ctx();
      if (n <= c.ell_cap && c.ell) return NCGPU_OK;
      if (c.ell) cudaFree(c.ell);
      if (c.ell_code) cudaFree(c.ell_code);
      if (c.ell_list) cudaFree(c.ell_list);
      c.ell = nullptr;
      c.ell_code = nullptr;
      c.ell_list = nullptr;
      c.ell_cap = 0;
      const size_t cap = std::max<size_t>(n, (size_t)c.n_max + 1);
      NCG_CK(cudaMalloc(&c.ell, 16 * cap * sizeof(double)));
      NCG_CK(cudaMalloc(&c.ell_code, cap));
      NCG_CK(cudaMalloc(&c.ell_list, (2 * cap + 1) * sizeof(int)));
      c.ell_cap = cap;
      return NCGPU_OK;
}

}  // namespace
}  // namespace ncg

extern "C" int ncgpu_elliptic_begin(double mu, double *yx, unsigned long yx_cap, int *n_bodies, int *host_idx,
                                    struct ncgpu_body *host_rec, int host_cap, int *n_host)
{
      Ctx &c = ctx();
      reset_launches();
      c.ell_n = -1;
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      if (!yx || !n_bodies || !n_host || host_cap < 0 || (host_cap > 0 && (!host_idx || !host_rec)))
            return NCGPU_E_ARG;
      cudaStream_t st = c.s;
      int n = 0;
      NCG_TRY(compact_existing(c.ex, c.largest_id, &n, st));
      *n_bodies = n;
      *n_host = 0;
      if (2ul * (unsigned long)n > yx_cap) return NCGPU_E_CAPACITY;
      NCG_TRY(ensure_ell((size_t)n));
      const size_t N = c.ell_cap;
      double *ell = c.ell, *dyx = c.ell + 6 * N, *hrec = c.ell + 8 * N;
      int *list = c.ell_list, *slots = c.ell_list + 1 + N;
      NCG_CK(cudaMemsetAsync(list, 0, sizeof(int), st));
      const bool j2 = c.P.par_J2_bool && c.P.par_central_mass_bool;
      if (n > 0) {
            k_cart2ell<<<(n + 255) / 256, 256, 0, st>>>(state_view(), c.cm, c.cidx, n, mu, c.P.par_G,
                                                         c.P.par_central_mass_bool ? 1 : 0, j2 ? 1 : 0, c.j2,
                                                         c.P.par_R_unit, ell, (long)N, dyx, c.ell_code, list);
            NCG_LAUNCHED();
      }
      int nh = 0;
      NCG_CK(cudaMemcpyAsync(&nh, list, sizeof(int), cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaStreamSynchronize(st));
      *n_host = nh;
      if (nh > host_cap) return NCGPU_E_CAPACITY;
      if (nh > 0) {  // in slot order, as display()'s loop meets them
            std::vector<int> h((size_t)nh);
            NCG_CK(cudaMemcpyAsync(h.data(), list + 1, sizeof(int) * nh, cudaMemcpyDeviceToHost, st));
            NCG_CK(cudaStreamSynchronize(st));
            std::sort(h.begin(), h.end());
            NCG_CK(cudaMemcpyAsync(list + 1, h.data(), sizeof(int) * nh, cudaMemcpyHostToDevice, st));
            k_ell_gather<<<(nh + 255) / 256, 256, 0, st>>>(state_view(), c.cidx, list + 1, nh, hrec, slots);
            NCG_LAUNCHED();
            NCG_CK(cudaMemcpyAsync(host_rec, hrec, sizeof(double) * 8 * nh, cudaMemcpyDeviceToHost, st));
            NCG_CK(cudaMemcpyAsync(host_idx, slots, sizeof(int) * nh, cudaMemcpyDeviceToHost, st));
      }
      if (n > 0) NCG_CK(cudaMemcpyAsync(yx, dyx, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaStreamSynchronize(st));
      c.ell_n = n;
      c.ell_nhost = nh;
      c.ell_done = 0;
      return NCGPU_OK;
}

extern "C" int ncgpu_format_elliptic(const double *F, const double *host_alkhqp, int n_host, int mass_radius,
                                     char *text, unsigned long cap, unsigned long *lens)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded || c.ell_n < 0) return NCGPU_E_STATE;
      const int n = c.ell_n;
      if (!text || !lens || n_host != c.ell_nhost || (n > 0 && !F) || (n_host > 0 && !host_alkhqp))
            return NCGPU_E_ARG;
      cudaStream_t st = c.s;
      const size_t N = c.ell_cap;
      if (!c.ell_done) {
            double *ell = c.ell, *dF = c.ell + 6 * N, *halk = c.ell + 8 * N;
            if (n > 0) {
                  NCG_CK(cudaMemcpyAsync(dF, F, sizeof(double) * n, cudaMemcpyHostToDevice, st));
                  k_ell_lambda<<<(n + 255) / 256, 256, 0, st>>>(dF, c.ell_code, ell + N, n);
                  NCG_LAUNCHED();
            }
            if (n_host > 0) {
                  NCG_CK(cudaMemcpyAsync(halk, host_alkhqp, sizeof(double) * 6 * n_host, cudaMemcpyHostToDevice, st));
                  k_ell_host<<<(n_host + 255) / 256, 256, 0, st>>>(c.ell_list + 1, halk, n_host, ell, (long)N);
                  NCG_LAUNCHED();
            }
            c.ell_done = 1;
      }
      const long first[9] = {0, n, 2L * n, 3L * n, 4L * n, 5L * n, 6L * n, 7L * n, 8L * n};
      // the element blocks are N apart: format them from a compact view
      return format_files(EllValues{state_view(), c.ell, c.cidx, n, (long)N}, mass_radius ? 8 : 6, first, text, cap,
                          lens);
}

extern "C" int ncgpu_elliptic_values(double *values, unsigned long cap)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded || c.ell_n < 0 || !c.ell_done) return NCGPU_E_STATE;
      if (!values) return NCGPU_E_ARG;
      const int n = c.ell_n;
      if (8ul * (unsigned long)n > cap) return NCGPU_E_CAPACITY;
      cudaStream_t st = c.s;
      const size_t N = c.ell_cap;
      for (int f = 0; f < 6 && n > 0; f++)
            NCG_CK(cudaMemcpyAsync(values + (size_t)f * n, c.ell + f * N, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                   st));
      if (n > 0) {  // masses and radii, gathered through the compacted slots
            double *g = c.ell + 8 * N;
            k_gather_mass<<<(n + 255) / 256, 256, 0, st>>>(state_view(), c.cidx, n, g);
            NCG_LAUNCHED();
            NCG_CK(cudaMemcpyAsync(values + 6 * (size_t)n, g, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
            k_gather_radius<<<(n + 255) / 256, 256, 0, st>>>(state_view(), c.cidx, n, g + N);
            NCG_LAUNCHED();
            NCG_CK(cudaMemcpyAsync(values + 7 * (size_t)n, g + N, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
      }
      NCG_CK(cudaStreamSynchronize(st));
      return NCGPU_OK;
}

extern "C" int ncgpu_host_atan2(const double *yx, double *F, long n)
{
      if (n < 0 || (n > 0 && (!yx || !F))) return NCGPU_E_ARG;
      const long per = 1L << 16;
      const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
      const int T = (int)std::min<long>(std::min<long>(hw, 16), (n + per - 1) / per);
      auto run = [&](long lo, long hi) {
            for (long j = lo; j < hi; j++) F[j] = atan2(yx[2 * j], yx[2 * j + 1]);
      };
      if (T <= 1) {
            run(0, n);
            return NCGPU_OK;
      }
      std::vector<std::thread> th;
      const long chunk = (n + T - 1) / T;
      for (int t = 0; t < T; t++) th.emplace_back(run, std::min(n, t * chunk), std::min(n, (t + 1) * chunk));
      for (auto &x : th) x.join();
      return NCGPU_OK;
}

extern "C" int ncgpu_output_stats(double *stats, int *idx, struct ncgpu_body *cm, struct ncgpu_body *two)
{
      Ctx &c = ctx();
      const int pre = c.stats_pre;  // started by ncgpu_format_cartesian just before
      c.stats_pre = 0;
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      if (!stats || !idx || !cm || !two) return NCGPU_E_ARG;
      cudaStream_t st = c.s;
      if (pre) {
            NCG_CK(cudaStreamWaitEvent(st, c.sev1, 0));
      } else {
            int n = 0;
            NCG_TRY(compact_existing(c.ex, c.largest_id, &n, st));
            NCG_TRY(stats_launch(n, st));
      }
      const double *res = c.red + 3900;
      const int *didx = (const int *)(c.red + 3904);
      int hidx[2];
      NCG_CK(cudaMemcpyAsync(stats, res, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaMemcpyAsync(hidx, didx, sizeof hidx, cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaMemcpyAsync(cm, c.cm, 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaStreamSynchronize(st));
      idx[0] = hidx[0];
      idx[1] = hidx[1];
      // the two bodies' records (slot 0's when absent, as the reference reads it)
      const double *fld[8] = {c.x, c.y, c.z, c.vx, c.vy, c.vz, c.m, c.R};
      for (int k = 0; k < 2; k++)
            for (int f = 0; f < 8; f++)
                  NCG_CK(cudaMemcpyAsync((double *)&two[k] + f, fld[f] + hidx[k], sizeof(double), cudaMemcpyDeviceToHost,
                                         st));
      NCG_CK(cudaStreamSynchronize(st));
      return NCGPU_OK;
}
