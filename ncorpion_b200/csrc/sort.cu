// Order-preserving primitives: stream compaction of existing slots and a
// stable LSD radix sort of (uint32 key, int value) pairs.  Both are used by the
// tiled gravity (space-filling-curve ordering) and the mesh search (sort of
// bodies by mesh cell, which replaces the reference's hash-table chains,
// src/structure.c:577-610 and :712-841).
#include "common.cuh"

namespace ncg {

namespace {

constexpr int CB = 1024;  // compaction block (one slot per thread)

__global__ void k_count_flags(const int *__restrict__ ex, int n, int *__restrict__ cnt)
{
      int i = blockIdx.x * CB + threadIdx.x;
      int f = (i < n && ex[i] != 0) ? 1 : 0;
      int c = __syncthreads_count(f);
      if (threadIdx.x == 0) cnt[blockIdx.x] = c;
}

// Exclusive scan of a[0..n) in place with one block of 1024 threads; writes
// the total to *total.
__global__ void k_scan_single(int *__restrict__ a, int n, int *__restrict__ total)
{
      __shared__ int part[1024];
      int t = threadIdx.x;
      int seg = (n + 1023) / 1024;
      int lo = t * seg, hi = min(n, lo + seg);
      int s = 0;
      for (int i = lo; i < hi; i++) s += a[i];
      part[t] = s;
      __syncthreads();
      for (int off = 1; off < 1024; off <<= 1) {
            int v = t >= off ? part[t - off] : 0;
            __syncthreads();
            part[t] += v;
            __syncthreads();
      }
      int run = part[t] - s;  // exclusive prefix of this segment
      for (int i = lo; i < hi; i++) {
            int v = a[i];
            a[i] = run;
            run += v;
      }
      if (t == 1023) *total = part[1023];
}

__global__ void k_scatter_flags(const int *__restrict__ ex, int n, const int *__restrict__ off,
                                int *__restrict__ out)
{
      __shared__ int wsum[CB / 32];
      int i = blockIdx.x * CB + threadIdx.x;
      int f = (i < n && ex[i] != 0) ? 1 : 0;
      unsigned b = __ballot_sync(0xffffffffu, f);
      int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
      int r = __popc(b & ((1u << lane) - 1u));
      if (lane == 0) wsum[w] = __popc(b);
      __syncthreads();
      if (threadIdx.x < 32) {
            int v = wsum[threadIdx.x];
            for (int o = 1; o < 32; o <<= 1) {
                  int u = __shfl_up_sync(0xffffffffu, v, o);
                  if (threadIdx.x >= o) v += u;
            }
            wsum[threadIdx.x] = v - wsum[threadIdx.x];
      }
      __syncthreads();
      if (f) out[off[blockIdx.x] + wsum[w] + r] = i;
}

// ---- radix sort -------------------------------------------------------------
constexpr int RT = 256;           // threads per block
constexpr int RK = 8;             // keys per thread (large sorts; small ones take fewer, RK_ template)
constexpr int RADIX = 256;

// Per-block digit counts: hist[digit][block] (digit-major, the order of the
// global offsets a scan gives), or hist[block][digit] when block_major (read by
// k_radix_scatter_inline, one coalesced row per block).
template <int RK_>
__global__ void k_radix_hist(const uint32_t *__restrict__ keys, int n, int shift,
                             int *__restrict__ hist, int nblocks, bool block_major)
{
      __shared__ int h[RADIX];
      h[threadIdx.x] = 0;
      __syncthreads();
      int base = blockIdx.x * RT * RK_;
#pragma unroll
      for (int r = 0; r < RK_; r++) {
            int i = base + r * RT + threadIdx.x;
            if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xffu], 1);
      }
      __syncthreads();
      hist[block_major ? blockIdx.x * RADIX + threadIdx.x : threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

template <int RK_>
__global__ void k_radix_scatter(const uint32_t *__restrict__ kin, const int *__restrict__ vin,
                                uint32_t *__restrict__ kout, int *__restrict__ vout, int n,
                                int shift, const int *__restrict__ hist, int nblocks)
{
      __shared__ int run[RADIX];
      __shared__ int gofs[RADIX];
      __shared__ int wc[RT / 32][RADIX];
      int t = threadIdx.x, lane = t & 31, w = t >> 5;
      run[t] = 0;
      gofs[t] = hist[t * nblocks + blockIdx.x];
      int base = blockIdx.x * RT * RK_;
      // the thread's keys and values of all rounds, loaded up front (independent loads)
      uint32_t kr[RK_];
      int vr[RK_];
#pragma unroll
      for (int r = 0; r < RK_; r++) {
            const int i = base + r * RT + t;
            kr[r] = i < n ? kin[i] : 0u;
            vr[r] = i < n ? vin[i] : 0;
      }
#pragma unroll
      for (int r = 0; r < RK_; r++) {
            for (int q = 0; q < RT / 32; q++) wc[q][t] = 0;
            __syncthreads();
            const int i = base + r * RT + t;
            const uint32_t key = kr[r];
            const int val = vr[r];
            const int d = i < n ? (int)((key >> shift) & 0xffu) : RADIX;  // RADIX: no key
            unsigned peers = __match_any_sync(0xffffffffu, d);
            int rk = __popc(peers & ((1u << lane) - 1u));
            int leader = __ffs(peers) - 1;
            if (lane == leader && d < RADIX) wc[w][d] = __popc(peers);
            __syncthreads();
            {
                  int acc = run[t];
#pragma unroll
                  for (int q = 0; q < RT / 32; q++) {
                        int c = wc[q][t];
                        wc[q][t] = acc;
                        acc += c;
                  }
                  run[t] = acc;
            }
            __syncthreads();
            if (d < RADIX) {
                  int dst = gofs[d] + wc[w][d] + rk;
                  kout[dst] = key;
                  vout[dst] = val;
            }
            __syncthreads();
      }
}

// k_radix_scatter for up to 128 blocks: each block finds its
// digits' global offsets from the unscanned histograms itself (the totals of
// every digit over all blocks, scanned across the block's 256 threads, plus the
// counts of the blocks before it), which saves the histogram scan's launches.
template <int RK_>
__global__ void k_radix_scatter_inline(const uint32_t *__restrict__ kin, const int *__restrict__ vin,
                                       uint32_t *__restrict__ kout, int *__restrict__ vout, int n, int shift,
                                       const int *__restrict__ hist, int nblocks)
{
      __shared__ int run[RADIX];
      __shared__ int gofs[RADIX];
      __shared__ int wc[RT / 32][RADIX];
      __shared__ int wsum[RT / 32];
      int t = threadIdx.x, lane = t & 31, w = t >> 5;
      int tot = 0, pre = 0;
#pragma unroll 8
      for (int b = 0; b < nblocks; b++) {  // block-major: one coalesced row per block
            const int v = hist[b * RADIX + t];
            tot += v;
            if (b < (int)blockIdx.x) pre += v;
      }
      int x = tot;  // exclusive scan of the digit totals over the 256 digits
      for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += u;
      }
      if (lane == 31) wsum[w] = x;
      __syncthreads();
      int before = 0;
      for (int q = 0; q < w; q++) before += wsum[q];
      gofs[t] = before + x - tot + pre;
      run[t] = 0;
      int base = blockIdx.x * RT * RK_;
      // the thread's keys and values of all rounds, loaded up front (independent loads)
      uint32_t kr[RK_];
      int vr[RK_];
#pragma unroll
      for (int r = 0; r < RK_; r++) {
            const int i = base + r * RT + t;
            kr[r] = i < n ? kin[i] : 0u;
            vr[r] = i < n ? vin[i] : 0;
      }
#pragma unroll
      for (int r = 0; r < RK_; r++) {
            for (int q = 0; q < RT / 32; q++) wc[q][t] = 0;
            __syncthreads();
            const int i = base + r * RT + t;
            const uint32_t key = kr[r];
            const int val = vr[r];
            const int d = i < n ? (int)((key >> shift) & 0xffu) : RADIX;  // RADIX: no key
            unsigned peers = __match_any_sync(0xffffffffu, d);
            int rk = __popc(peers & ((1u << lane) - 1u));
            int leader = __ffs(peers) - 1;
            if (lane == leader && d < RADIX) wc[w][d] = __popc(peers);
            __syncthreads();
            {
                  int acc = run[t];
#pragma unroll
                  for (int q = 0; q < RT / 32; q++) {
                        int c = wc[q][t];
                        wc[q][t] = acc;
                        acc += c;
                  }
                  run[t] = acc;
            }
            __syncthreads();
            if (d < RADIX) {
                  int dst = gofs[d] + wc[w][d] + rk;
                  kout[dst] = key;
                  vout[dst] = val;
            }
            __syncthreads();
      }
}

// Exclusive scan of one 1024-element block; block total to sums[b].
__global__ void k_block_scan(const int *__restrict__ in, int n, int *__restrict__ out, int *__restrict__ sums)
{
      __shared__ int ws[32];
      int i = blockIdx.x * 1024 + threadIdx.x;
      int v = i < n ? in[i] : 0;
      int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
      int x = v;
      for (int o = 1; o < 32; o <<= 1) {
            int u = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += u;
      }
      if (lane == 31) ws[w] = x;
      __syncthreads();
      if (w == 0) {
            int y = ws[lane];
            for (int o = 1; o < 32; o <<= 1) {
                  int u = __shfl_up_sync(0xffffffffu, y, o);
                  if (lane >= o) y += u;
            }
            ws[lane] = y;
      }
      __syncthreads();
      int excl = x - v + (w > 0 ? ws[w - 1] : 0);
      if (i < n) out[i] = excl;
      if (threadIdx.x == 1023) sums[blockIdx.x] = ws[31];
}

__global__ void k_add_block_offsets(int *__restrict__ out, int n, const int *__restrict__ sums)
{
      int i = blockIdx.x * 1024 + threadIdx.x;
      if (i < n) out[i] += sums[blockIdx.x];
}

}  // namespace

// out[i] = sum of in[0..i); out[n] = total (out has n + 1 entries).
// `sums` is scratch of at least ceil(n / 1024) + 1 ints.
int scan_exclusive(const int *in, int *out, int n, int *sums, cudaStream_t st)
{
      if (n <= 0) {
            NCG_CK(cudaMemsetAsync(out, 0, sizeof(int), st));
            return NCGPU_OK;
      }
      int nb = (n + 1023) / 1024;
      k_block_scan<<<nb, 1024, 0, st>>>(in, n, out, sums);
      NCG_LAUNCHED();
      k_scan_single<<<1, 1024, 0, st>>>(sums, nb, out + n);
      NCG_LAUNCHED();
      k_add_block_offsets<<<nb, 1024, 0, st>>>(out, n, sums);
      NCG_LAUNCHED();
      return NCGPU_OK;
}

int compact_existing_dev(const int *ex, int largest_id, cudaStream_t st)
{
      Ctx &c = ctx();
      int n = largest_id + 1;
      if (n <= 0) {
            NCG_CK(cudaMemsetAsync(c.n_dev, 0, sizeof(int), st));
            return NCGPU_OK;
      }
      int nb = (n + CB - 1) / CB;
      k_count_flags<<<nb, CB, 0, st>>>(ex, n, c.cnt);
      NCG_LAUNCHED();
      k_scan_single<<<1, 1024, 0, st>>>(c.cnt, nb, c.n_dev);
      NCG_LAUNCHED();
      k_scatter_flags<<<nb, CB, 0, st>>>(ex, n, c.cnt, c.cidx);
      NCG_LAUNCHED();
      return NCGPU_OK;
}

int compact_existing(const int *ex, int largest_id, int *n_host, cudaStream_t st)
{
      Ctx &c = ctx();
      int n = largest_id + 1;
      if (n <= 0) {
            *n_host = 0;
            return NCGPU_OK;
      }
      int nb = (n + CB - 1) / CB;
      k_count_flags<<<nb, CB, 0, st>>>(ex, n, c.cnt);
      NCG_LAUNCHED();
      k_scan_single<<<1, 1024, 0, st>>>(c.cnt, nb, c.n_dev);
      NCG_LAUNCHED();
      k_scatter_flags<<<nb, CB, 0, st>>>(ex, n, c.cnt, c.cidx);
      NCG_LAUNCHED();
      NCG_CK(cudaMemcpyAsync(n_host, c.n_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaStreamSynchronize(st));
      return NCGPU_OK;
}

int radix_sort_pairs(uint32_t *keys, int *vals, int n, int bits, cudaStream_t st)
{
      Ctx &c = ctx();
      if (n <= 1) return NCGPU_OK;
      // keys per thread: the fewest (1, 2, 4) that keep a small sort within 128
      // blocks, else 8; up to 128 blocks the scatter scans the histograms itself
      // (two launches a pass), beyond that a scan runs between the two kernels
      int kpt = RK;
      for (int k = 1; k < RK; k <<= 1)
            if ((n + RT * k - 1) / (RT * k) <= 128) {
                  kpt = k;
                  break;
            }
      const int nb = (n + RT * kpt - 1) / (RT * kpt);
      size_t need = (size_t)RADIX * nb;
      if (need > c.hist_cap) return NCGPU_E_CAPACITY;
      uint32_t *ka = keys, *kb = c.keys2;
      int *va = vals, *vb = c.vals2;
      if (keys == c.keys2 || vals == c.vals2) return NCGPU_E_ARG;
      int passes = (bits + 7) / 8;
      for (int p = 0; p < passes; p++) {
            int shift = 8 * p;
#define NCG_RADIX_PASS(K)                                                                       \
      do {                                                                                      \
            k_radix_hist<K><<<nb, RT, 0, st>>>(ka, n, shift, c.hist, nb, nb <= 128);           \
            NCG_LAUNCHED();                                                                     \
            if (nb <= 128) {                                                                    \
                  k_radix_scatter_inline<K><<<nb, RT, 0, st>>>(ka, va, kb, vb, n, shift, c.hist, nb); \
            } else {                                                                            \
                  NCG_TRY(scan_exclusive(c.hist, c.hist, (int)need, c.cnt, st));                \
                  k_radix_scatter<K><<<nb, RT, 0, st>>>(ka, va, kb, vb, n, shift, c.hist, nb);  \
            }                                                                                   \
            NCG_LAUNCHED();                                                                     \
      } while (0)
            if (kpt == 1) NCG_RADIX_PASS(1);
            else if (kpt == 2) NCG_RADIX_PASS(2);
            else if (kpt == 4) NCG_RADIX_PASS(4);
            else NCG_RADIX_PASS(RK);
#undef NCG_RADIX_PASS
            uint32_t *tk = ka; ka = kb; kb = tk;
            int *tv = va; va = vb; vb = tv;
      }
      if (ka != keys) {  // odd number of passes: result is in the scratch pair
            NCG_CK(cudaMemcpyAsync(keys, ka, sizeof(uint32_t) * (size_t)n, cudaMemcpyDeviceToDevice, st));
            NCG_CK(cudaMemcpyAsync(vals, va, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, st));
      }
      return NCGPU_OK;
}

}  // namespace ncg

namespace ncg {

// Order-preserving compaction of the flagged slots 0..n_slots-1 into out_idx
// with caller-provided scratch (blockcnt: ceil(n_slots/1024) + 1 ints, n_dev:
// 1 int); the count is copied to *n_host (synchronises the stream).
int compact_flags_into(const int *flags, int n_slots, int *blockcnt, int *n_dev, int *out_idx, int *n_host,
                       cudaStream_t st)
{
      if (n_slots <= 0) {
            *n_host = 0;
            return NCGPU_OK;
      }
      int nb = (n_slots + CB - 1) / CB;
      k_count_flags<<<nb, CB, 0, st>>>(flags, n_slots, blockcnt);
      NCG_LAUNCHED();
      k_scan_single<<<1, 1024, 0, st>>>(blockcnt, nb, n_dev);
      NCG_LAUNCHED();
      k_scatter_flags<<<nb, CB, 0, st>>>(flags, n_slots, blockcnt, out_idx);
      NCG_LAUNCHED();
      NCG_CK(cudaMemcpyAsync(n_host, n_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaStreamSynchronize(st));
      return NCGPU_OK;
}

}  // namespace ncg
