// An allocation-free variant of the exact gravity evaluation.
//
// Some callers cannot allocate device memory at the point where they need a
// force evaluation: a host whose device memory is fully handed to its own pool
// allocator before the integration starts, or a real-time or latency-bound
// integration loop that forbids allocation (and the synchronisation it
// implies) once it runs.  ncgpu_vector_field_static serves them: it needs no
// ncgpu_init, allocates nothing (no cudaMalloc, cudaFree or allocating library
// call), and keeps its scratch in the fixed file-scope device array below.
//
// The array belongs to the library's device code: every GPU that loads that
// code holds NOALLOC_SCRATCH_BYTES of it until the process exits.  CUDA loads
// device code lazily by default (CUDA_MODULE_LOADING=LAZY), so the array and
// the kernels reach a device at the first call on that device, not when the
// library is opened.  The first call on each device is therefore the set-up:
// with that device current it loads the code and the array, and resolves the
// array's device address with cudaGetSymbolAddress (host code cannot use the
// array's name as a device address: on the host it is only a stand-in).  Make
// that first call before the host's pool allocator takes the device's memory
// and before any stream capture, or run with CUDA_MODULE_LOADING=EAGER.  The
// address is cached per device under a lock; cudaDeviceReset invalidates it,
// so a process that resets a device must not call this entry point again.
// All calls share the one array and it keeps the last call's contents: what
// must start at zero is cleared at every call, and calls that overlap on the
// GPU (other streams, other host threads) race on it.
#include <string.h>
#include <mutex>
#include "common.cuh"

namespace ncg {
namespace {

constexpr int NOALLOC_MAX_SLOTS = NCGPU_NOALLOC_MAX_SLOTS;
constexpr size_t NPAD = ((size_t)NOALLOC_MAX_SLOTS + 127) / 128 * 128;
constexpr size_t NBLK = (size_t)NOALLOC_MAX_SLOTS / 1024 + 2;

// layout (doubles first, 256-byte aligned blocks)
constexpr size_t OFF_SRC = 0;                                   // 4 * NPAD doubles
constexpr size_t OFF_SRCR = OFF_SRC + 4 * NPAD * 8;             // NPAD doubles
constexpr size_t OFF_CTERM = OFF_SRCR + NPAD * 8;               // 6 * NPAD doubles (two per body with J2)
constexpr size_t OFF_ACC = OFF_CTERM + 6 * NPAD * 8;            // 3 * NPAD doubles
constexpr size_t OFF_CIDX = OFF_ACC + 3 * NPAD * 8;             // NPAD ints
constexpr size_t OFF_BLK = OFF_CIDX + NPAD * 4;                 // NBLK ints
constexpr size_t OFF_MISC = (OFF_BLK + NBLK * 4 + 255) / 256 * 256;  // n_dev, err
constexpr size_t NOALLOC_SCRATCH_BYTES = OFF_MISC + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
static unsigned char *g_scratch_addr[MAX_DEVICES];
static std::mutex g_scratch_lock;

// The device address of g_noalloc_scratch on the current device, resolved at
// the first call on that device and cached (a failed lookup is retried).
int scratch_address(unsigned char **out)
{
      int dev = 0;
      NCG_CK(cudaGetDevice(&dev));
      if (dev < 0 || dev >= MAX_DEVICES) return NCGPU_E_UNSUPPORTED;
      std::lock_guard<std::mutex> hold(g_scratch_lock);
      if (!g_scratch_addr[dev]) {
            void *p = nullptr;
            NCG_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
            g_scratch_addr[dev] = (unsigned char *)p;
      }
      *out = g_scratch_addr[dev];
      return NCGPU_OK;
}

}  // namespace
}  // namespace ncg

using namespace ncg;

extern "C" unsigned long ncgpu_noalloc_scratch_bytes(void) { return (unsigned long)NOALLOC_SCRATCH_BYTES; }

extern "C" int ncgpu_vector_field_static(const double *d_bodies, const int *d_exists, int largest_id,
                                         const struct ncgpu_body *cm, const struct ncgpu_params *params,
                                         double *d_acc, double *d_cm_acc, void *stream)
{
      reset_launches();
      if (!d_bodies || !d_exists || !cm || !params || !d_acc || !d_cm_acc) return NCGPU_E_ARG;
      if (largest_id < -1) return NCGPU_E_ARG;
      if (largest_id + 1 > NOALLOC_MAX_SLOTS) return NCGPU_E_CAPACITY;  // beyond the static scratch
      unsigned char *base = nullptr;
      NCG_TRY(scratch_address(&base));
      cudaStream_t st = (cudaStream_t)stream;
      double *src = (double *)(base + OFF_SRC), *srcR = (double *)(base + OFF_SRCR);
      double *cterm = (double *)(base + OFF_CTERM), *acc = (double *)(base + OFF_ACC);
      int *cidx = (int *)(base + OFF_CIDX), *blk = (int *)(base + OFF_BLK);
      int *n_dev = (int *)(base + OFF_MISC);
      unsigned *err = (unsigned *)(base + OFF_MISC + 64);
      NCG_CK(cudaMemsetAsync(base + OFF_BLK, 0, OFF_MISC + 256 - OFF_BLK, st));  // counts, n, error word
      BodyView bv{d_bodies, d_bodies + 1, d_bodies + 2, d_bodies + 3, d_bodies + 4, d_bodies + 5,
                  d_bodies + 6, d_bodies + 7, 8, d_exists};
      const long bs = largest_id + 1;
      if (params->par_J2_bool && !params->par_central_mass_bool) return NCGPU_E_ARG;
      NCG_TRY(gravity_exact_into(bv, largest_id, (const double *)cm, params->par_G, params->par_softening_parameter,
                                 params->par_central_mass_bool, j2_arg(*params, cm->mass, j2_value(*params, cm->mass, params->par_sideral_omega)), cidx, src, srcR, cterm,
                                 blk, n_dev, err, acc,
                                 acc + NPAD, acc + 2 * NPAD, d_cm_acc, st));
      if (bs > 0) {
            for (int d = 0; d < 3; d++)
                  NCG_CK(cudaMemcpy2DAsync(d_acc + d, 3 * sizeof(double), acc + d * NPAD, sizeof(double),
                                           sizeof(double), bs, cudaMemcpyDeviceToDevice, st));
      }
      unsigned h = 0;
      NCG_CK(cudaMemcpyAsync(&h, err, sizeof h, cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaStreamSynchronize(st));
      if (h & ERR_TIMEOUT) return NCGPU_E_TIMEOUT;
      if (h) return NCGPU_E_CUDA;
      return NCGPU_OK;
}
