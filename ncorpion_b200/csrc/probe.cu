// Diagnostic FP32 throughput probes: independent FFMA chains (scalar and the
// sm_100a packed f32x2 form) and independent rsqrt.approx chains, with enough
// warps per SM to saturate each pipe.  The measured rates are the denominators
// of the FP32 gravity kernel's roofline fractions.
#include "common.cuh"
#include "bulk.cuh"

namespace ncg {
namespace {

constexpr int PROBE_ITERS = 4096;

__global__ void __launch_bounds__(256) k_ffma_probe(float *out, float a, float b)
{
      float r0 = threadIdx.x * 1e-7f, r1 = r0 + 1.f, r2 = r0 + 2.f, r3 = r0 + 3.f;
      float r4 = r0 + 4.f, r5 = r0 + 5.f, r6 = r0 + 6.f, r7 = r0 + 7.f;
#pragma unroll 4
      for (int i = 0; i < PROBE_ITERS; i++) {
            r0 = fmaf(r0, a, b); r1 = fmaf(r1, a, b); r2 = fmaf(r2, a, b); r3 = fmaf(r3, a, b);
            r4 = fmaf(r4, a, b); r5 = fmaf(r5, a, b); r6 = fmaf(r6, a, b); r7 = fmaf(r7, a, b);
      }
      float s = ((r0 + r1) + (r2 + r3)) + ((r4 + r5) + (r6 + r7));
      if (s == 123.456f) out[0] = s;  // keeps the chains live
}

__global__ void __launch_bounds__(256) k_ffma2_probe(float *out, float a, float b)
{
      unsigned long long A, B, r[8];
      asm("mov.b64 %0, {%1, %1};" : "=l"(A) : "f"(a));
      asm("mov.b64 %0, {%1, %1};" : "=l"(B) : "f"(b));
      for (int k = 0; k < 8; k++) {
            const float lo = threadIdx.x * 1e-7f + k, hi = lo + 0.5f;
            asm("mov.b64 %0, {%1, %2};" : "=l"(r[k]) : "f"(lo), "f"(hi));
      }
#pragma unroll 4
      for (int i = 0; i < PROBE_ITERS; i++) {
#pragma unroll
            for (int k = 0; k < 8; k++) asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(r[k]) : "l"(A), "l"(B));
      }
      float s = 0.f;
      for (int k = 0; k < 8; k++) {
            float lo, hi;
            asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(r[k]));
            s += lo + hi;
      }
      if (s == 123.456f) out[0] = s;
}

__global__ void __launch_bounds__(256) k_rsqrt_probe(float *out, float b)
{
      float r[8];
      for (int k = 0; k < 8; k++) r[k] = 1.f + threadIdx.x * 1e-7f + k;
#pragma unroll 4
      for (int i = 0; i < PROBE_ITERS; i++) {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                  float y;
                  asm volatile("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(r[k]));
                  r[k] = y + b;  // stays near 1: alternates around the fixed point
            }
      }
      float s = 0.f;
      for (int k = 0; k < 8; k++) s += r[k];
      if (s == 123.456f) out[0] = s;
}

// One thread waits on an mbarrier that nothing will complete, for at most
// `probes` failed try_waits (the primitive of every bounded wait here), then
// records the timeout in the error word as the real kernels do, with the
// cycles the wait took.
__global__ void k_timeout_probe(int probes, unsigned *err, long long *cycles)
{
      __shared__ uint64_t bar;
      if (threadIdx.x != 0) return;
      mbar_init(&bar, 1);
      mbar_fence_init();
      const long long t0 = clock64();
      bool ok = false;
      for (int it = 0; it < probes && !ok; ++it) ok = mbar_try_wait(&bar, 0);
      *cycles = clock64() - t0;
      if (!ok) atomicOr(err, ERR_TIMEOUT);
}

}  // namespace
}  // namespace ncg

using namespace ncg;

namespace {
// Best-of-5 duration (ms) of one probe launch over sms*8 blocks of 256 threads.
template <typename L>
int best_ms(L launch, float *best)
{
      cudaEvent_t e0, e1;
      NCG_CK(cudaEventCreate(&e0));
      NCG_CK(cudaEventCreate(&e1));
      launch();  // warm-up
      NCG_LAUNCHED();
      *best = 1e30f;
      for (int rep = 0; rep < 5; rep++) {
            NCG_CK(cudaEventRecord(e0));
            launch();
            NCG_LAUNCHED();
            NCG_CK(cudaEventRecord(e1));
            NCG_CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            NCG_CK(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < *best) *best = ms;
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return NCGPU_OK;
}
}  // namespace

extern "C" int ncgpu_probe_fp32_rates(double *ffma_tflops, double *ffma2_tflops, double *rsqrt_gops)
{
      if (!ffma_tflops || !ffma2_tflops || !rsqrt_gops) return NCGPU_E_ARG;
      int dev = 0, sms = 0;
      NCG_CK(cudaGetDevice(&dev));
      NCG_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      float *out = nullptr;
      NCG_CK(cudaMalloc(&out, sizeof(float)));
      const int blocks = sms * 8;
      const double lanes = (double)blocks * 256.0 * 8.0 * PROBE_ITERS;
      float ms = 0.f;
      int st = best_ms([&] { k_ffma_probe<<<blocks, 256>>>(out, 0.9999f, 1e-6f); }, &ms);
      if (st == NCGPU_OK) {
            *ffma_tflops = 2.0 * lanes / (ms * 1e-3) / 1e12;
            st = best_ms([&] { k_ffma2_probe<<<blocks, 256>>>(out, 0.9999f, 1e-6f); }, &ms);
      }
      if (st == NCGPU_OK) {
            *ffma2_tflops = 4.0 * lanes / (ms * 1e-3) / 1e12;
            st = best_ms([&] { k_rsqrt_probe<<<blocks, 256>>>(out, 0.5f); }, &ms);
      }
      if (st == NCGPU_OK) *rsqrt_gops = lanes / (ms * 1e-3) / 1e9;
      cudaFree(out);
      return st;
}

extern "C" int ncgpu_probe_fp32_peak(double *tflops)
{
      if (!tflops) return NCGPU_E_ARG;
      int dev = 0, sms = 0;
      NCG_CK(cudaGetDevice(&dev));
      NCG_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      float *out = nullptr;
      NCG_CK(cudaMalloc(&out, sizeof(float)));
      cudaEvent_t e0, e1;
      NCG_CK(cudaEventCreate(&e0));
      NCG_CK(cudaEventCreate(&e1));
      const int blocks = sms * 8;
      k_ffma_probe<<<blocks, 256>>>(out, 0.9999f, 1e-6f);  // warm-up
      NCG_LAUNCHED();
      float best = 1e30f;
      for (int rep = 0; rep < 5; rep++) {
            NCG_CK(cudaEventRecord(e0));
            k_ffma_probe<<<blocks, 256>>>(out, 0.9999f, 1e-6f);
            NCG_LAUNCHED();
            NCG_CK(cudaEventRecord(e1));
            NCG_CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            NCG_CK(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < best) best = ms;
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      cudaFree(out);
      double flops = 2.0 * 8.0 * PROBE_ITERS * (double)blocks * 256.0;
      *tflops = flops / (best * 1e-3) / 1e12;
      return NCGPU_OK;
}

extern "C" int ncgpu_probe_wait_timeout(int probes, double *cycles_per_probe)
{
      Ctx &c = ctx();
      reset_launches();
      if (!c.inited) return NCGPU_E_STATE;
      if (probes < 1 || probes > WAIT_LIMIT || !cycles_per_probe) return NCGPU_E_ARG;
      long long *cyc = (long long *)c.n_dev;  // 8 spare bytes of the library's scratch ints
      k_timeout_probe<<<1, 32, 0, c.s>>>(probes, c.err, cyc);
      NCG_LAUNCHED();
      long long h = 0;
      NCG_CK(cudaMemcpyAsync(&h, cyc, sizeof h, cudaMemcpyDeviceToHost, c.s));
      NCG_CK(cudaStreamSynchronize(c.s));
      *cycles_per_probe = (double)h / probes;
      return check_err_word();
}

namespace ncg {
namespace {
__global__ void k_div_probe(const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ out,
                            int n)
{
      const int i = blockIdx.x * blockDim.x + threadIdx.x;
      if (i < n) out[i] = div_by_recip(a[i], b[i], __drcp_rn(b[i]));
}
}  // namespace
}  // namespace ncg

// out[i] = a[i] / b[i] through div_by_recip (the quotient of the tides'
// recurrence), for tests against correctly rounded division.  Host buffers.
extern "C" int ncgpu_probe_div(const double *a, const double *b, double *out, int n)
{
      if (!a || !b || !out || n <= 0) return NCGPU_E_ARG;
      double *d = nullptr;
      NCG_CK(cudaMalloc(&d, 3 * sizeof(double) * (size_t)n));
      NCG_CK(cudaMemcpy(d, a, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice));
      NCG_CK(cudaMemcpy(d + n, b, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice));
      k_div_probe<<<(n + 255) / 256, 256>>>(d, d + n, d + 2 * (size_t)n, n);
      NCG_LAUNCHED();
      NCG_CK(cudaMemcpy(out, d + 2 * (size_t)n, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost));
      NCG_CK(cudaFree(d));
      return NCGPU_OK;
}

namespace ncg {
namespace {
// out[c] = s0[c] + x[c*n] + ... + x[c*n + n-1], one warp per chain, by the
// run-taking sum (runs != 0) or the plain staged loop.
__global__ void __launch_bounds__(RUN_NW * 32) k_seq_probe(const double *__restrict__ x, long n,
                                                           const double *__restrict__ s0, double *__restrict__ out,
                                                           int runs)
{
      extern __shared__ __align__(16) double stage[];  // RUN_STAGE doubles
      const int c = blockIdx.x;
      const double *t = x + (size_t)c * n;
      if (runs) {
            const double s = block_run_sum(t, n, s0[c], stage);
            if (threadIdx.x == 0) out[c] = s;
      } else if (threadIdx.x < 32) {
            const double s = warp_chain_sum(t, n, s0[c], stage);
            if (threadIdx.x == 0) out[c] = s;
      }
}
}  // namespace
}  // namespace ncg

extern "C" int ncgpu_probe_seq_sum(const double *x, long n, const double *s0, double *out, int chains, int runs)
{
      if (!x || !s0 || !out || n < 0 || chains <= 0 || chains > 65535) return NCGPU_E_ARG;
      const size_t nx = (size_t)n * (size_t)chains;
      double *d = nullptr;
      NCG_CK(cudaMalloc(&d, sizeof(double) * (nx + 2 * (size_t)chains)));
      if (nx) NCG_CK(cudaMemcpy(d, x, sizeof(double) * nx, cudaMemcpyHostToDevice));
      NCG_CK(cudaMemcpy(d + nx, s0, sizeof(double) * (size_t)chains, cudaMemcpyHostToDevice));
      constexpr int smem = ncg::RUN_STAGE * (int)sizeof(double);
      NCG_CK(cudaFuncSetAttribute(ncg::k_seq_probe, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      ncg::k_seq_probe<<<chains, ncg::RUN_NW * 32, smem>>>(d, n, d + nx, d + nx + chains, runs);
      NCG_LAUNCHED();
      NCG_CK(cudaMemcpy(out, d + nx + chains, sizeof(double) * (size_t)chains, cudaMemcpyDeviceToHost));
      NCG_CK(cudaFree(d));
      return NCGPU_OK;
}
