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
#include "common.cuh"

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

// Value j of file f (0..5: x y z vx vy vz with the central body first when
// `central`; 6, 7: mass and radius of the bodies only).
__device__ __forceinline__ double out_value(const BodyView &S, const double *cm, const int *cidx, int central, int f,
                                            int j)
{
      const int c = f < 6 ? central : 0;
      if (j < c) return cm[f];
      const long s = (long)cidx[j - c] * S.stride;
      const double *a[8] = {S.x, S.y, S.z, S.vx, S.vy, S.vz, S.m, S.R};
      return a[f][s];
}

// One thread per value: formatted into its slot, the length into len.
__global__ void k_fmt_values(BodyView S, const double *__restrict__ cm, const int *__restrict__ cidx, int n,
                             int central, char *__restrict__ slots, int *__restrict__ len, unsigned *err)
{
      const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
      const int per = n + central;  // values in files 0..5
      const long total = 6L * per + 2L * n;
      if (i >= total) return;
      int f, j;
      if (i < 6L * per) {
            f = (int)(i / per);
            j = (int)(i % per);
      } else {
            f = 6 + (int)((i - 6L * per) / n);
            j = (int)((i - 6L * per) % n);
      }
      const int L = fmt_fixed14(out_value(S, cm, cidx, central, f, j), slots + (size_t)i * SLOT);
      if (L < 0) atomicOr(err, ERR_INTERNAL);
      len[i] = L < 0 ? 0 : L;
}

// Copies the slots to their places in the packed text (offsets: exclusive
// scan of the lengths; the files' texts follow one another, without newlines).
__global__ void k_fmt_pack(const char *__restrict__ slots, const int *__restrict__ off, long total,
                           char *__restrict__ text)
{
      const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
      if (i >= total) return;
      const int L = off[i + 1] - off[i];
      const char *src = slots + (size_t)i * SLOT;
      char *dst = text + off[i];
      for (int c = 0; c < L; c++) dst[c] = src[c];
}

// display()'s statistics of the bodies (src/display.c:303-379): the total mass,
// summed in slot order, and the two most massive bodies as its loop picks them
// (strictly greater replaces, so the first of equal masses wins; i1 = i2 = 0 and
// M = 0 when there are fewer positive masses).  One warp.
__global__ void k_out_stats(BodyView S, const int *__restrict__ cidx, int n, double *__restrict__ out_mass,
                            int *__restrict__ out_idx)
{
      // per lane, then merged: the first (m desc, slot asc) and the first of the
      // others; only positive masses take part (the loop starts from M = 0)
      double M1 = 0., M2 = 0.;
      int i1 = 0x7fffffff, i2 = 0x7fffffff;
      for (int q = threadIdx.x; q < n; q += 32) {
            const int p = cidx[q];  // ascending within a lane
            const double m = S.m[(long)p * S.stride];
            if (m > M1) { M2 = M1; i2 = i1; M1 = m; i1 = p; }
            else if (m > M2) { M2 = m; i2 = p; }
      }
      for (int o = 16; o > 0; o >>= 1) {
            double a1 = M1, a2 = M2, b1 = __shfl_xor_sync(0xffffffffu, M1, o), b2 = __shfl_xor_sync(0xffffffffu, M2, o);
            int j1 = i1, j2 = i2, k1 = __shfl_xor_sync(0xffffffffu, i1, o), k2 = __shfl_xor_sync(0xffffffffu, i2, o);
            if (b1 > a1 || (b1 == a1 && k1 < j1)) {  // the other list leads
                  double t = a1; a1 = b1; b1 = t; t = a2; a2 = b2; b2 = t;
                  int u = j1; j1 = k1; k1 = u; u = j2; j2 = k2; k2 = u;
            }
            const bool bsec = b1 > a2 || (b1 == a2 && k1 < j2);  // second: the better of a2 and b1
            M1 = a1; i1 = j1;
            M2 = bsec ? b1 : a2;
            i2 = bsec ? k1 : j2;
      }
      if (threadIdx.x == 0) {
            out_mass[1] = M1;
            out_mass[2] = M2;
            out_idx[0] = M1 > 0. ? i1 : 0;
            out_idx[1] = M2 > 0. ? i2 : 0;
      }
}

__global__ void k_gather_mass(BodyView S, const int *__restrict__ cidx, int n, double *__restrict__ m)
{
      const int q = blockIdx.x * blockDim.x + threadIdx.x;
      if (q < n) m[q] = S.m[(long)cidx[q] * S.stride];
}

__global__ void __launch_bounds__(32) k_chain_total(const double *__restrict__ m, int n, double *__restrict__ out)
{
      __shared__ __align__(16) double stage[CHN];
      const double s = warp_chain_sum(m, n, 0., stage);
      if (threadIdx.x == 0) out[0] = s;
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

extern "C" int ncgpu_format_cartesian(char *text, unsigned long cap, unsigned long *lens)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      if (!text || !lens) return NCGPU_E_ARG;
      cudaStream_t st = c.s;
      int n = 0;
      NCG_TRY(compact_existing(c.ex, c.largest_id, &n, st));
      const int central = c.P.par_central_mass_bool ? 1 : 0;
      const long per = n + central, total = 6 * per + 2L * n;
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
      BodyView S = state_view();
      int h[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      if (total > 0) {
            const int nb = (int)((total + 255) / 256);
            k_fmt_values<<<nb, 256, 0, st>>>(S, c.cm, c.cidx, n, central, c.fmt_slots, len, c.err);
            NCG_LAUNCHED();
            NCG_TRY(scan_exclusive(len, off, (int)total, sums, st));
            k_fmt_pack<<<nb, 256, 0, st>>>(c.fmt_slots, off, total, c.fmt_text);
            NCG_LAUNCHED();
            // each file's first value (files 0..5: per values; 6, 7: n values)
            const long first[9] = {0, per, 2 * per, 3 * per, 4 * per, 5 * per, 6 * per, 6 * per + n, total};
            for (int f = 0; f < 9; f++)
                  NCG_CK(cudaMemcpyAsync(&h[f], off + first[f], sizeof(int), cudaMemcpyDeviceToHost, st));
      }
      unsigned herr = 0;
      NCG_CK(cudaMemcpyAsync(&herr, c.err, sizeof herr, cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaStreamSynchronize(st));
      if (herr & ERR_INTERNAL) {  // a value beyond the formatter's range
            NCG_CK(cudaMemsetAsync(c.err, 0, sizeof(unsigned), st));
            return NCGPU_E_UNSUPPORTED;
      }
      if (herr) return check_err_word();
      if ((unsigned long)h[8] > cap) return NCGPU_E_CAPACITY;
      if (h[8] > 0) {
            NCG_CK(cudaMemcpyAsync(text, c.fmt_text, (size_t)h[8], cudaMemcpyDeviceToHost, st));
            NCG_CK(cudaStreamSynchronize(st));
      }
      for (int f = 0; f < 8; f++) lens[f] = (unsigned long)(h[f + 1] - h[f]);
      return NCGPU_OK;
}

extern "C" int ncgpu_output_stats(double *stats, int *idx, struct ncgpu_body *cm, struct ncgpu_body *two)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      if (!stats || !idx || !cm || !two) return NCGPU_E_ARG;
      cudaStream_t st = c.s;
      int n = 0;
      NCG_TRY(compact_existing(c.ex, c.largest_id, &n, st));
      NCG_TRY(ensure_partial((size_t)n + 8));
      BodyView S = state_view();
      double *m = c.partial, *res = c.red + 3900;
      int *didx = (int *)(c.red + 3904);
      if (n > 0) {
            k_gather_mass<<<(n + 255) / 256, 256, 0, st>>>(S, c.cidx, n, m);
            NCG_LAUNCHED();
      }
      k_chain_total<<<1, 32, 0, st>>>(m, n, res);
      NCG_LAUNCHED();
      k_out_stats<<<1, 32, 0, st>>>(S, c.cidx, n, res, didx);
      NCG_LAUNCHED();
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
