// C-ABI entry points of libncgpu: context lifetime, state transfer, the
// stateless vector_field replacement and the leapfrog kick / drift.
#include <string.h>
#include <stdlib.h>
#include <algorithm>
#include "common.cuh"

namespace ncg {

static Ctx g_ctx;
static char g_last_error[512] = "";
static int g_launches = 0;

Ctx &ctx() { return g_ctx; }

int cuda_fail(cudaError_t e, const char *what, const char *file, int line)
{
      snprintf(g_last_error, sizeof g_last_error, "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
      return NCGPU_E_CUDA;
}
void note_launch() { ++g_launches; }
void reset_launches()
{
      g_launches = 0;
      if (g_ctx.stats_pre) {  // statistics still running on the second stream: later work waits for them
            cudaStreamWaitEvent(g_ctx.s, g_ctx.sev1, 0);
            g_ctx.stats_pre = 0;
      }
}
int launches() { return g_launches; }

int ensure_partial(size_t doubles)
{
      Ctx &c = ctx();
      if (doubles <= c.partial_cap) return NCGPU_OK;
      if (c.partial) NCG_CK(cudaFree(c.partial));
      c.partial = nullptr;
      c.partial_cap = 0;
      NCG_CK(cudaMalloc(&c.partial, doubles * sizeof(double)));
      c.partial_cap = doubles;
      return NCGPU_OK;
}

int check_err_word()
{
      Ctx &c = ctx();
      unsigned h = 0;
      NCG_CK(cudaMemcpyAsync(&h, c.err, sizeof h, cudaMemcpyDeviceToHost, c.s));
      NCG_CK(cudaStreamSynchronize(c.s));
      if (h) NCG_CK(cudaMemsetAsync(c.err, 0, sizeof(unsigned), c.s));
      if (h & ERR_TIMEOUT) return NCGPU_E_TIMEOUT;
      if (h & ERR_NMAX) return NCGPU_E_NMAX;
      if (h & ERR_FRAGMENT) return NCGPU_E_FRAGMENT;
      if (h & ERR_CAPACITY) return NCGPU_E_CAPACITY;
      if (h) return NCGPU_E_CUDA;
      return NCGPU_OK;
}

namespace {

template <class Tp>
int dalloc(Tp **p, size_t count)
{
      NCG_CK(cudaMalloc((void **)p, count * sizeof(Tp)));
      return NCGPU_OK;
}

}  // namespace
void mesh_free();
namespace {

void free_all()
{
      Ctx &c = ctx();
      mesh_free();
      void *ptrs[] = {c.x, c.y, c.z, c.vx, c.vy, c.vz, c.m, c.R, c.ex, c.cm, c.cm_acc, c.acc, c.cmterm,
                      c.partial, c.cidx, c.cnt, c.n_dev, c.src64, c.srcR, c.src32, c.srcR32, c.tilebox,
                      c.keys, c.keys2, c.vals, c.vals2, c.hist, c.red, c.err, c.aos, c.exs,
                      c.did, c.dirty, c.dlist, c.free_idx, c.scal, c.hi, c.hj, c.ev, c.evrec,
                      c.snap[0], c.snap[1], c.snap[2], c.snap[3], c.snap[4], c.snap[5], c.snap[6], c.snap[7],
                      c.snap_cm, c.fmt_slots, c.fmt_text, c.fmt_len, c.ell, c.ell_code, c.ell_list, c.lf_buf};
      for (void *p : ptrs)
            if (p) cudaFree(p);
      if (c.pinned) cudaFreeHost(c.pinned);
      if (c.kev0) cudaEventDestroy(c.kev0);
      if (c.kev1) cudaEventDestroy(c.kev1);
      if (c.sev0) cudaEventDestroy(c.sev0);
      if (c.sev1) cudaEventDestroy(c.sev1);
      if (c.s2) cudaStreamDestroy(c.s2);
      if (c.cev) cudaEventDestroy(c.cev);
      if (c.s3) cudaStreamDestroy(c.s3);
      if (c.s) cudaStreamDestroy(c.s);
      c = Ctx{};
}

__global__ void k_aos_to_soa(const double *__restrict__ aos, int n, double *x, double *y, double *z, double *vx,
                             double *vy, double *vz, double *m, double *R)
{
      int i = blockIdx.x * blockDim.x + threadIdx.x;
      if (i >= n) return;
      const double *b = aos + 8 * (size_t)i;
      x[i] = b[0]; y[i] = b[1]; z[i] = b[2];
      vx[i] = b[3]; vy[i] = b[4]; vz[i] = b[5];
      m[i] = b[6]; R[i] = b[7];
}

// The accelerations of the existing bodies into the velocity fields of the
// device copy of the caller's records (the other fields keep the bytes the
// caller sent), so that one contiguous copy returns them.
__global__ void k_acc_into_aos(double *__restrict__ aos, const int *__restrict__ ex, int n,
                               const double *__restrict__ ax, const double *__restrict__ ay,
                               const double *__restrict__ az)
{
      int i = blockIdx.x * blockDim.x + threadIdx.x;
      if (i >= n || !ex[i]) return;
      double *b = aos + 8 * (size_t)i;
      b[3] = ax[i]; b[4] = ay[i]; b[5] = az[i];
}

__global__ void k_soa_to_aos(double *__restrict__ aos, int n, const double *x, const double *y, const double *z,
                             const double *vx, const double *vy, const double *vz, const double *m, const double *R)
{
      int i = blockIdx.x * blockDim.x + threadIdx.x;
      if (i >= n) return;
      double *b = aos + 8 * (size_t)i;
      b[0] = x[i]; b[1] = y[i]; b[2] = z[i];
      b[3] = vx[i]; b[4] = vy[i]; b[5] = vz[i];
      b[6] = m[i]; b[7] = R[i];
}

// (ax, ay, az) blocks -> xyz triples out[3k + d]
__global__ void k_interleave3(const double *__restrict__ ax, const double *__restrict__ ay,
                              const double *__restrict__ az, long n, double *__restrict__ out)
{
      const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
      if (k >= n) return;
      out[3 * k] = ax[k];
      out[3 * k + 1] = ay[k];
      out[3 * k + 2] = az[k];
}

// kick, src/rk4.c:96-105: v += timestep * a for existing bodies, then the
// central mass with CM_acc.  Explicit _rn operations: no FMA contraction.
__global__ void k_kick(const int *__restrict__ ex, int n, double dt, const double *__restrict__ ax,
                       const double *__restrict__ ay, const double *__restrict__ az, double *vx, double *vy,
                       double *vz, double *cm, const double *__restrict__ cm_acc, int kick_cm)
{
      int i = blockIdx.x * blockDim.x + threadIdx.x;
      if (i < n && ex[i]) {
            vx[i] = __dadd_rn(vx[i], __dmul_rn(dt, ax[i]));
            vy[i] = __dadd_rn(vy[i], __dmul_rn(dt, ay[i]));
            vz[i] = __dadd_rn(vz[i], __dmul_rn(dt, az[i]));
      }
      if (i == 0 && kick_cm) {
            cm[3] = __dadd_rn(cm[3], __dmul_rn(dt, cm_acc[0]));
            cm[4] = __dadd_rn(cm[4], __dmul_rn(dt, cm_acc[1]));
            cm[5] = __dadd_rn(cm[5], __dmul_rn(dt, cm_acc[2]));
      }
}

// drift, src/rk4.c:115-126: x += timestep * v.
__global__ void k_drift(const int *__restrict__ ex, int n, double dt, double *x, double *y, double *z,
                        const double *__restrict__ vx, const double *__restrict__ vy,
                        const double *__restrict__ vz, double *cm, int drift_cm)
{
      int i = blockIdx.x * blockDim.x + threadIdx.x;
      if (i < n && ex[i]) {
            x[i] = __dadd_rn(x[i], __dmul_rn(dt, vx[i]));
            y[i] = __dadd_rn(y[i], __dmul_rn(dt, vy[i]));
            z[i] = __dadd_rn(z[i], __dmul_rn(dt, vz[i]));
      }
      if (i == 0 && drift_cm) {
            cm[0] = __dadd_rn(cm[0], __dmul_rn(dt, cm[3]));
            cm[1] = __dadd_rn(cm[1], __dmul_rn(dt, cm[4]));
            cm[2] = __dadd_rn(cm[2], __dmul_rn(dt, cm[5]));
      }
}

}  // namespace

BodyView state_view()
{
      Ctx &c = ctx();
      BodyView v{c.x, c.y, c.z, c.vx, c.vy, c.vz, c.m, c.R, 1, c.ex};
      return v;
}

int state_cm_host(double *cm9)
{
      Ctx &c = ctx();
      NCG_CK(cudaMemcpyAsync(cm9, c.cm, 9 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
      NCG_CK(cudaStreamSynchronize(c.s));
      return NCGPU_OK;
}

// The J2 in force for the state's kicks: J2_value, or the fluid-body J2 of the
// state's central mass and rotation at this moment, which is when the
// reference sets it (upload = variable_initialization, src/structure.c:507;
// end of a step, src/rk4.c:459-463).  Kicks between two updates use it even if
// the rotation changes meanwhile.
int refresh_j2()
{
      Ctx &c = ctx();
      if (!c.P.par_J2_bool) return NCGPU_OK;
      double cm9[9];
      NCG_TRY(state_cm_host(cm9));
      c.j2_prev = c.j2;
      c.j2 = j2_value(c.P, cm9[6], cm9[8]);
      return NCGPU_OK;
}

int mesh_gravity_state(const J2Arg &j2);

int kick_state()
{
      Ctx &c = ctx();
      c.com_reduced = 0;
      const int nslots = c.largest_id + 1;
      const bool mesh_grav = c.P.par_mesh_bool && !c.force_naive && !c.P.par_mesh_brute_gravity;
      // the central mass's state on the host: for the brute-force gravity's
      // arguments and the J2 term; mesh gravity, and the exact brute force on a
      // few thousand bodies, read it from device memory
      const bool exact_small = c.P.par_gravity_mode == NCGPU_GRAVITY_EXACT && nslots <= EXACT_SMALL_N;
      double cm9[9] = {0.};
      if ((!mesh_grav && !exact_small) || c.P.par_J2_bool) NCG_TRY(state_cm_host(cm9));
      const J2Arg j2 = j2_arg(c.P, cm9[6], c.j2);
      if (mesh_grav)
            NCG_TRY(mesh_gravity_state(j2));
      else
            NCG_TRY(gravity_eval(state_view(), c.largest_id, cm9, j2, c.acc, c.n_max, c.cm_acc, c.P.par_gravity_mode,
                                 c.s, 0, 1, c.cm));
      if (c.P.par_central_tides_bool && c.P.par_central_mass_bool) NCG_TRY(tides_state(c.acc, c.n_max, c.cm_acc));
      int nb = nslots > 0 ? (nslots + 255) / 256 : 1;
      k_kick<<<nb, 256, 0, c.s>>>(c.ex, nslots, c.dt, c.acc, c.acc + c.n_max, c.acc + 2 * (size_t)c.n_max, c.vx,
                                  c.vy, c.vz, c.cm, c.cm_acc, c.P.par_central_mass_bool);
      NCG_LAUNCHED();
      return NCGPU_OK;
}

int drift_state()
{
      Ctx &c = ctx();
      c.com_reduced = 0;
      const int nslots = c.largest_id + 1;
      int nb = nslots > 0 ? (nslots + 255) / 256 : 1;
      k_drift<<<nb, 256, 0, c.s>>>(c.ex, nslots, c.dt, c.x, c.y, c.z, c.vx, c.vy, c.vz, c.cm,
                                   c.P.par_central_mass_bool);
      NCG_LAUNCHED();
      return NCGPU_OK;
}

}  // namespace ncg

using namespace ncg;

extern "C" {

void ncgpu_default_params(struct ncgpu_params *p)
{
      if (!p) return;
      memset(p, 0, sizeof *p);
      p->par_G = 39.47841760435743447533796;  // src/parameters.h:131
      p->par_softening_parameter = 0.;
      p->par_central_mass_bool = 1;
      p->par_mutual_bool = 1;
      p->par_collision_bool = 1;
      p->par_brute_force_bool = 1;
      p->par_mesh_bool = 0;
      p->par_collision_type = NCGPU_COLLISION_MERGER;
      p->par_collision_parameter = 2.;
      p->par_one_collision_only_bool = 0;
      p->par_collision_cube_cells = 1024;
      p->par_how_many_neighbours = 16.;
      p->par_collision_cube_min = 80.;
      p->par_switch_to_brute_force = 110;
      p->par_gravity_mode = NCGPU_GRAVITY_EXACT;
      p->par_near_theta = 0.15;
      p->par_disruption_threshold = 1.8;     // src/parameters.h:150
      p->par_high_dumping_threshold = 230.95;  // src/parameters.h:177
      p->par_reduce_to_COM_bool = 1;
      p->par_N_tilde = 15;  // src/parameters.h:297-307
      p->par_pq_min_max[0] = -1;
      p->par_pq_min_max[1] = 3;
      p->par_pq_min_max[2] = -1;
      p->par_pq_min_max[3] = 1;
      p->par_mu_parameter = 0.55;
      p->par_nu_parameter = 0.4;
      p->par_C1_parameter = 1.5;
      p->par_k_parameter = 0.2;
      p->par_merging_threshold = 0.0002;
      p->par_fragment_threshold = 1.5e-8;
      p->par_mesh_brute_gravity = 0;
      p->par_J2_bool = 0;
      p->par_J2 = 0.;
      p->par_R_unit = 1.;
      p->par_sideral_omega = 2. * 3.14159265358979323846 / 3.556721809;  /* Tearth's default */
      p->par_central_tides_bool = 0;
      p->par_k2 = 1.5;                  /* src/parameters.h:143-145 */
      p->par_Delta_t = 0.0015807;
      p->par_dimensionless_moi = 0.3307;
}

const char *ncgpu_strerror(int s)
{
      switch (s) {
      case NCGPU_OK: return "ok";
      case NCGPU_E_ARG: return "bad argument";
      case NCGPU_E_CUDA: return "CUDA error";
      case NCGPU_E_CAPACITY: return "device buffer capacity exceeded";
      case NCGPU_E_NMAX: return "Cannot add a body to the simulation. Try increasing the value of N_max.";
      case NCGPU_E_STATE: return "library not initialised or state not uploaded";
      case NCGPU_E_TIMEOUT: return "device-side wait timed out";
      case NCGPU_E_UNSUPPORTED: return "configuration not supported by the GPU path";
      case NCGPU_E_FRAGMENT:
            return "Error: In function fragmentation, the velocity of a fragment cannot be less than the escape velocity.";
      default: return "unknown status";
      }
}

const char *ncgpu_last_error(void) { return g_last_error; }
int ncgpu_last_launch_count(void) { return launches(); }
void *ncgpu_stream(void) { return g_ctx.inited ? (void *)g_ctx.s : nullptr; }

// Parameter checks of the reference's own (src/structure.c:1278, 1407-1410)
// that concern the device path, plus the gravity mode's range.
static bool params_ok(const struct ncgpu_params *p)
{
      if (!p || p->par_gravity_mode < 0 || p->par_gravity_mode > 2) return false;
      if (p->par_J2_bool != 0 && p->par_J2_bool != 1) return false;
      if (p->par_central_tides_bool != 0 && p->par_central_tides_bool != 1) return false;
      if ((p->par_J2_bool || p->par_central_tides_bool) && !p->par_central_mass_bool) return false;
      return true;
}

int ncgpu_init(int n_max, const struct ncgpu_params *params)
{
      if (n_max <= 0 || !params_ok(params)) return NCGPU_E_ARG;
      if (g_ctx.inited) ncgpu_finalize();
      Ctx &c = g_ctx;
      c.P = *params;
      c.n_max = n_max;
      size_t N = (size_t)n_max;
      size_t npad = ((N + 127) / 128) * 128;
      int st = NCGPU_OK;
#define A(ptr, cnt)                                          \
      do {                                                   \
            if ((st = dalloc(&(ptr), (cnt))) != NCGPU_OK) {  \
                  free_all();                                \
                  return st;                                 \
            }                                                \
      } while (0)
      A(c.x, N); A(c.y, N); A(c.z, N); A(c.vx, N); A(c.vy, N); A(c.vz, N); A(c.m, N); A(c.R, N);
      A(c.ex, N); A(c.exs, N);
      A(c.cm, 16); A(c.cm_acc, 3);
      A(c.acc, 3 * N);
      A(c.cmterm, 6 * N);
      A(c.cidx, N);
      A(c.cnt, (std::max(N, (size_t)1 << 20) + 1023) / 1024 + 2);
      A(c.n_dev, 8);
      {
            double *p = nullptr;
            A(p, 4 * npad);
            c.src64 = p;
      }
      A(c.srcR, npad);
      {
            float *p = nullptr;
            A(p, 4 * npad);
            c.src32 = p;
      }
      {
            int dev = 0;
            NCG_CK(cudaGetDevice(&dev));
            NCG_CK(cudaDeviceGetAttribute(&c.sm_count, cudaDevAttrMultiProcessorCount, dev));
            const char *e = getenv("NCGPU_GRAV_SLOTS_MULT");
            if (e && atoi(e) > 0) c.grav_slots_mult = atoi(e);
      }
      A(c.srcR32, npad);
      A(c.tilebox, 6 * (npad / 128));
      // sort scratch: at least 2^20 keys, so collision-hit lists of dense
      // clusters sort even when n_max is small
      const size_t NS = std::max(N, (size_t)1 << 20);
      A(c.keys, NS); A(c.keys2, NS); A(c.vals, NS); A(c.vals2, NS);
      c.hist_cap = 256 * ((NS + 2047) / 2048);
      A(c.hist, c.hist_cap + 1);  // + total of the in-place scan
      A(c.red, 4096);
      A(c.err, 1);
      A(c.aos, 8 * N);
      A(c.did, N); A(c.dirty, N); A(c.dlist, 3 * N); A(c.free_idx, N); A(c.scal, S_COUNT);
      c.hit_cap = (int)NS;
      A(c.hi, NS); A(c.hj, NS);
      c.ev_cap = (int)(2 * N + 1024);
      A(c.ev, 3 * (size_t)c.ev_cap);
      A(c.evrec, EVREC * (size_t)c.ev_cap);
#undef A
      if (cudaMallocHost((void **)&c.pinned, 8 * N * sizeof(double)) != cudaSuccess) {
            free_all();
            return NCGPU_E_CUDA;
      }
      if (cudaEventCreate(&c.kev0) != cudaSuccess || cudaEventCreate(&c.kev1) != cudaSuccess) {
            free_all();
            return NCGPU_E_CUDA;
      }
      if (cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking) != cudaSuccess ||
          cudaStreamCreateWithFlags(&c.s2, cudaStreamNonBlocking) != cudaSuccess ||
          cudaStreamCreateWithFlags(&c.s3, cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&c.cev, cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&c.sev0, cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&c.sev1, cudaEventDisableTiming) != cudaSuccess) {
            free_all();
            return NCGPU_E_CUDA;
      }
      if ((st = ensure_partial(3 * std::max(npad, (size_t)4096 * 128))) != NCGPU_OK) {
            free_all();
            return st;
      }
      cudaMemsetAsync(c.err, 0, sizeof(unsigned), c.s);
      cudaMemsetAsync(c.ex, 0, N * sizeof(int), c.s);
      cudaMemsetAsync(c.did, 0, N * sizeof(int), c.s);
      cudaMemsetAsync(c.dirty, 0, N, c.s);
      cudaMemsetAsync(c.scal, 0, S_COUNT * sizeof(int), c.s);
      double cm0[16] = {0., 0., 0., 0., 0., 0., 1., 1., params->par_sideral_omega};
      cudaMemcpyAsync(c.cm, cm0, sizeof cm0, cudaMemcpyHostToDevice, c.s);
      c.j2 = j2_value(*params, 1., params->par_sideral_omega);
      if (cudaStreamSynchronize(c.s) != cudaSuccess) {
            free_all();
            return NCGPU_E_CUDA;
      }
      c.inited = 1;
      return NCGPU_OK;
}

int ncgpu_last_kernel_ms(double *ms)
{
      if (!ms) return NCGPU_E_ARG;
      if (!g_ctx.inited || !g_ctx.kev_valid) return NCGPU_E_STATE;
      NCG_CK(cudaEventSynchronize(g_ctx.kev1));
      float f = 0.f;
      NCG_CK(cudaEventElapsedTime(&f, g_ctx.kev0, g_ctx.kev1));
      *ms = f;
      return NCGPU_OK;
}

int ncgpu_set_params(const struct ncgpu_params *params)
{
      if (!g_ctx.inited) return NCGPU_E_STATE;
      if (!params_ok(params)) return NCGPU_E_ARG;
      g_ctx.P = *params;
      if (g_ctx.uploaded) return refresh_j2();
      return NCGPU_OK;
}

int ncgpu_host_register(void *ptr, unsigned long bytes)
{
      if (!ptr || bytes == 0) return NCGPU_E_ARG;
      NCG_CK(cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterDefault));
      return NCGPU_OK;
}

int ncgpu_host_unregister(void *ptr)
{
      if (!ptr) return NCGPU_E_ARG;
      NCG_CK(cudaHostUnregister(ptr));
      return NCGPU_OK;
}

void ncgpu_finalize(void)
{
      if (g_ctx.s) cudaStreamSynchronize(g_ctx.s);
      free_all();
}

int ncgpu_vector_field_dev(const double *d_bodies, const int *d_exists, int largest_id,
                           const struct ncgpu_body *cm, double *d_acc, double *d_cm_acc, int gravity_mode,
                           void *stream)
{
      return ncgpu_vector_field_part(d_bodies, d_exists, largest_id, cm, 0, 1, d_acc, d_cm_acc, gravity_mode, stream);
}

int ncgpu_vector_field_part(const double *d_bodies, const int *d_exists, int largest_id,
                            const struct ncgpu_body *cm, int part, int nparts, double *d_acc, double *d_cm_acc,
                            int gravity_mode, void *stream)
{
      Ctx &c = g_ctx;
      reset_launches();
      if (!c.inited) return NCGPU_E_STATE;
      if (!d_bodies || !d_exists || !cm || !d_acc || !d_cm_acc) return NCGPU_E_ARG;
      if (nparts < 1 || part < 0 || part >= nparts) return NCGPU_E_ARG;
      if (largest_id < -1 || largest_id >= c.n_max) return NCGPU_E_ARG;
      cudaStream_t st = stream ? (cudaStream_t)stream : c.s;
      BodyView bv{d_bodies, d_bodies + 1, d_bodies + 2, d_bodies + 3, d_bodies + 4, d_bodies + 5,
                  d_bodies + 6, d_bodies + 7, 8, d_exists};
      // d_acc is 3 consecutive blocks of (largest_id + 1) doubles
      long bs = largest_id + 1;
      // gravity_eval writes ax, ay, az blocks; repack to xyz triples
      const J2Arg j2 = j2_arg(c.P, cm->mass, j2_value(c.P, cm->mass, c.P.par_sideral_omega));
      NCG_TRY(gravity_eval(bv, largest_id, (const double *)cm, j2, c.acc, c.n_max, d_cm_acc, gravity_mode, st, part,
                           nparts));
      if (bs > 0) {  // interleave into d_acc[3*k + d]
            k_interleave3<<<(int)((bs + 255) / 256), 256, 0, st>>>(c.acc, c.acc + c.n_max, c.acc + 2 * (size_t)c.n_max,
                                                                  bs, d_acc);
            NCG_LAUNCHED();
      }
      return NCGPU_OK;
}

int ncgpu_check_error(void *stream)
{
      Ctx &c = g_ctx;
      if (!c.inited) return NCGPU_E_STATE;
      if (stream) NCG_CK(cudaStreamSynchronize((cudaStream_t)stream));
      return check_err_word();
}

int ncgpu_vector_field(struct ncgpu_body *bodies, const int *exists, int largest_id, const struct ncgpu_body *cm,
                       double *cm_acc, int gravity_mode)
{
      Ctx &c = g_ctx;
      reset_launches();
      if (!c.inited) return NCGPU_E_STATE;
      if (!bodies || !exists || !cm || !cm_acc) return NCGPU_E_ARG;
      if (largest_id < -1 || largest_id >= c.n_max) return NCGPU_E_ARG;
      const int ns = largest_id + 1;
      cudaStream_t st = c.s;
      if (ns > 0) {
            NCG_CK(cudaMemcpyAsync(c.aos, bodies, sizeof(struct ncgpu_body) * (size_t)ns, cudaMemcpyHostToDevice, st));
            NCG_CK(cudaMemcpyAsync(c.exs, exists, sizeof(int) * (size_t)ns, cudaMemcpyHostToDevice, st));
      }
      BodyView bv{c.aos, c.aos + 1, c.aos + 2, c.aos + 3, c.aos + 4, c.aos + 5, c.aos + 6, c.aos + 7, 8, c.exs};
      const J2Arg j2 = j2_arg(c.P, cm->mass, j2_value(c.P, cm->mass, c.P.par_sideral_omega));
      NCG_TRY(gravity_eval(bv, largest_id, (const double *)cm, j2, c.acc, c.n_max, c.cm_acc, gravity_mode, st));
      // the records come back whole: the velocity fields of the existing bodies
      // carry their accelerations, every other byte is the caller's own
      if (ns > 0) {
            k_acc_into_aos<<<(ns + 255) / 256, 256, 0, st>>>(c.aos, c.exs, ns, c.acc, c.acc + c.n_max,
                                                            c.acc + 2 * (size_t)c.n_max);
            NCG_LAUNCHED();
            NCG_CK(cudaMemcpyAsync(bodies, c.aos, sizeof(struct ncgpu_body) * (size_t)ns, cudaMemcpyDeviceToHost, st));
      }
      double *h = c.pinned;
      NCG_CK(cudaMemcpyAsync(h, c.cm_acc, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaStreamSynchronize(st));
      NCG_TRY(check_err_word());
      cm_acc[0] = h[0];
      cm_acc[1] = h[1];
      cm_acc[2] = h[2];
      return NCGPU_OK;
}

int ncgpu_upload(const struct ncgpu_body *bodies, const int *exists, int largest_id, const struct ncgpu_body *cm)
{
      Ctx &c = g_ctx;
      reset_launches();
      if (!c.inited) return NCGPU_E_STATE;
      if ((!bodies && largest_id >= 0) || (!exists && largest_id >= 0) || !cm) return NCGPU_E_ARG;
      if (largest_id < -1 || largest_id >= c.n_max) return NCGPU_E_ARG;
      const int ns = largest_id + 1;
      cudaStream_t st = c.s;
      NCG_CK(cudaMemsetAsync(c.ex, 0, sizeof(int) * (size_t)c.n_max, st));
      if (ns > 0) {
            NCG_CK(cudaMemcpyAsync(c.aos, bodies, sizeof(struct ncgpu_body) * (size_t)ns, cudaMemcpyHostToDevice, st));
            NCG_CK(cudaMemcpyAsync(c.ex, exists, sizeof(int) * (size_t)ns, cudaMemcpyHostToDevice, st));
            k_aos_to_soa<<<(ns + 255) / 256, 256, 0, st>>>(c.aos, ns, c.x, c.y, c.z, c.vx, c.vy, c.vz, c.m, c.R);
            NCG_LAUNCHED();
      }
      NCG_CK(cudaMemcpyAsync(c.cm, cm, 8 * sizeof(double), cudaMemcpyHostToDevice, st));
      NCG_CK(cudaMemsetAsync(c.did, 0, sizeof(int) * (size_t)c.n_max, st));
      int sc[S_COUNT] = {0};
      sc[S_LID] = largest_id;
      NCG_CK(cudaMemcpyAsync(c.scal, sc, sizeof sc, cudaMemcpyHostToDevice, st));
      NCG_CK(cudaStreamSynchronize(st));
      c.largest_id = largest_id;
      c.n_events = 0;
      c.collision_count = 0;
      c.uploaded = 1;
      c.com_reduced = 0;
      NCG_TRY(refresh_j2());
      c.j2_prev = c.j2;
      return NCGPU_OK;
}

int ncgpu_download(struct ncgpu_body *bodies, int *exists, int *largest_id, struct ncgpu_body *cm)
{
      Ctx &c = g_ctx;
      reset_launches();
      if (!c.inited || !c.uploaded) return NCGPU_E_STATE;
      if (!bodies || !exists || !largest_id || !cm) return NCGPU_E_ARG;
      const int ns = c.largest_id + 1;
      cudaStream_t st = c.s;
      if (ns > 0) {
            k_soa_to_aos<<<(ns + 255) / 256, 256, 0, st>>>(c.aos, ns, c.x, c.y, c.z, c.vx, c.vy, c.vz, c.m, c.R);
            NCG_LAUNCHED();
            NCG_CK(cudaMemcpyAsync(bodies, c.aos, sizeof(struct ncgpu_body) * (size_t)ns, cudaMemcpyDeviceToHost, st));
            NCG_CK(cudaMemcpyAsync(exists, c.ex, sizeof(int) * (size_t)ns, cudaMemcpyDeviceToHost, st));
      }
      NCG_CK(cudaMemcpyAsync(cm, c.cm, 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
      NCG_CK(cudaStreamSynchronize(st));
      *largest_id = c.largest_id;
      return check_err_word();
}

int ncgpu_get_j2(double *j2, double *j2_before)
{
      Ctx &c = g_ctx;
      if (!c.inited) return NCGPU_E_STATE;
      if (!j2) return NCGPU_E_ARG;
      *j2 = c.P.par_J2_bool ? c.j2 : 0.;
      if (j2_before) *j2_before = c.P.par_J2_bool ? c.j2_prev : 0.;
      return NCGPU_OK;
}

int ncgpu_get_sideral_omega(double *omega)
{
      Ctx &c = g_ctx;
      if (!c.inited) return NCGPU_E_STATE;
      if (!omega) return NCGPU_E_ARG;
      NCG_CK(cudaMemcpyAsync(omega, c.cm + 8, sizeof(double), cudaMemcpyDeviceToHost, c.s));
      NCG_CK(cudaStreamSynchronize(c.s));
      return NCGPU_OK;
}

int ncgpu_set_sideral_omega(double omega)
{
      Ctx &c = g_ctx;
      if (!c.inited) return NCGPU_E_STATE;
      NCG_CK(cudaMemcpyAsync(c.cm + 8, &omega, sizeof(double), cudaMemcpyHostToDevice, c.s));
      NCG_CK(cudaStreamSynchronize(c.s));
      return NCGPU_OK;
}

int ncgpu_set_timestep(double dt)
{
      if (!g_ctx.inited) return NCGPU_E_STATE;
      g_ctx.dt = dt;
      return NCGPU_OK;
}

int ncgpu_kick(void)
{
      reset_launches();
      if (!g_ctx.inited || !g_ctx.uploaded) return NCGPU_E_STATE;
      NCG_TRY(kick_state());
      return check_err_word();
}

int ncgpu_set_force_naive(int on)
{
      if (!g_ctx.inited) return NCGPU_E_STATE;
      g_ctx.force_naive = on ? 1 : 0;
      return NCGPU_OK;
}

int ncgpu_drift(void)
{
      reset_launches();
      if (!g_ctx.inited || !g_ctx.uploaded) return NCGPU_E_STATE;
      NCG_TRY(drift_state());
      return NCGPU_OK;
}

}  // extern "C"
