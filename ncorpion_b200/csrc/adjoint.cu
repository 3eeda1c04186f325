// Differentiable gravity + leapfrog: forward integration and its hand-written
// adjoint (reverse mode), no collisions.  There is no reference counterpart for
// the adjoint; the forward is the brute-force driver of the reference
// (src/rk4.c:873-936 with collision_bool = 0): half drift, then n x (kick with
// vector_field, drift), then the half back-drift of the final output, with the
// central mass integrated as a body (kick with CM_acc, drift).
//
// For body k and source j, r = x_j - x_k, D^2 = |r|^2 + eps_kj^2
// (eps_kj = softening_parameter * (R_k + R_j)), a_k = sum_j G m_j r / D^3.
// Tidal tensor T_kj = I/D^3 - 3 r r^T / D^5 (symmetric in k, j).
// Vector-Jacobian products with adjoint velocities lambda (bodies) and Lambda
// (central mass), central-mass offsets s_k = x_k - X, J_k = I/|s|^3 - 3 s s^T/|s|^5:
//   (da/dx)^T lambda |_k  = sum_j G T_kj (m_k lambda_j - m_j lambda_k)
//                           + G J_k (m_k Lambda - M lambda_k)
//   (da/dX)^T ...          = sum_k G J_k (M lambda_k - m_k Lambda)
//   (da/dm)^T ...     |_k  = -sum_j G (lambda_j . r) / D^3 + G Lambda . s_k / |s_k|^3
// Pair sums are FP64 with one rsqrt per pair, tiled through shared memory with
// (target block, source chunk) work units reduced in a fixed order.
#include "common.cuh"

namespace ncg {

namespace {

constexpr int AT = 128;  // bodies per tile / threads per block

struct Src {
      const double *x, *y, *z, *m, *sR, *lx, *ly, *lz;  // lx.. : adjoints (VJP) or position tangents (JVP)
      const double *dm;                                 // mass tangents (JVP)
};

// Mutual forces (OP 0: 3 outputs), their VJP (OP 1: 4 outputs) or their JVP
// (OP 2: 3 outputs, d a_k = sum_j G [dm_j r + m_j T_kj (dx_j - dx_k)] / ...)
// of target block blockIdx.y against source chunk blockIdx.x.
template <int OP, bool SOFT>
__global__ void __launch_bounds__(AT) k_pairs(Src s, int n, int tpc, double *__restrict__ part, long stride)
{
      __shared__ double sx[AT], sy[AT], sz[AT], sm[AT], sr[AT], slx[AT], sly[AT], slz[AT], sdm[AT];
      const int k = blockIdx.y * AT + threadIdx.x;
      const bool act = k < n;
      const int kk = act ? k : 0;
      const double xk = s.x[kk], yk = s.y[kk], zk = s.z[kk], mk = s.m[kk], rk = SOFT ? s.sR[kk] : 0.;
      double lxk = 0., lyk = 0., lzk = 0.;
      if (OP >= 1) { lxk = s.lx[kk]; lyk = s.ly[kk]; lzk = s.lz[kk]; }
      double o0 = 0., o1 = 0., o2 = 0., o3 = 0.;
      const int ntiles = (n + AT - 1) / AT;
      const int t0 = blockIdx.x * tpc, t1 = min(ntiles, t0 + tpc);
      for (int t = t0; t < t1; ++t) {
            const int j = t * AT + threadIdx.x;
            __syncthreads();
            if (j < n) {
                  sx[threadIdx.x] = s.x[j]; sy[threadIdx.x] = s.y[j]; sz[threadIdx.x] = s.z[j];
                  sm[threadIdx.x] = s.m[j];
                  if (SOFT) sr[threadIdx.x] = s.sR[j];
                  if (OP >= 1) { slx[threadIdx.x] = s.lx[j]; sly[threadIdx.x] = s.ly[j]; slz[threadIdx.x] = s.lz[j]; }
                  if (OP == 2) sdm[threadIdx.x] = s.dm[j];
            }
            __syncthreads();
            const int cnt = min(AT, n - t * AT);
            for (int q = 0; q < cnt; ++q) {
                  if (t * AT + q == k) continue;
                  const double rx = sx[q] - xk, ry = sy[q] - yk, rz = sz[q] - zk;
                  double d2 = 0.;
                  if (SOFT) { const double e = rk + sr[q]; d2 = e * e; }
                  d2 = fma(rx, rx, fma(ry, ry, fma(rz, rz, d2)));
                  const double ri = rsqrt(d2);
                  const double i3 = ri * ri * ri;
                  if (OP == 0) {
                        const double w = sm[q] * i3;
                        o0 = fma(w, rx, o0); o1 = fma(w, ry, o1); o2 = fma(w, rz, o2);
                  } else if (OP == 2) {
                        const double i5 = i3 * ri * ri;
                        const double dx = slx[q] - lxk, dy = sly[q] - lyk, dz = slz[q] - lzk;
                        const double rd = rx * dx + ry * dy + rz * dz;
                        const double mj = sm[q], c = 3.0 * rd * i5 * mj, g = sdm[q] * i3;
                        o0 += g * rx + mj * i3 * dx - rx * c;
                        o1 += g * ry + mj * i3 * dy - ry * c;
                        o2 += g * rz + mj * i3 * dz - rz * c;
                  } else {
                        const double i5 = i3 * ri * ri;
                        const double mj = sm[q];
                        const double wx = mk * slx[q] - mj * lxk, wy = mk * sly[q] - mj * lyk, wz = mk * slz[q] - mj * lzk;
                        const double rw = rx * wx + ry * wy + rz * wz;
                        const double c = 3.0 * rw * i5;
                        o0 += wx * i3 - rx * c; o1 += wy * i3 - ry * c; o2 += wz * i3 - rz * c;
                        o3 -= (slx[q] * rx + sly[q] * ry + slz[q] * rz) * i3;
                  }
            }
      }
      if (act) {
            double *p = part + (size_t)blockIdx.x * (OP == 1 ? 4 : 3) * stride;
            p[k] = o0; p[stride + k] = o1; p[2 * stride + k] = o2;
            if (OP == 1) p[3 * stride + k] = o3;
      }
}

}  // namespace

namespace {

// acc = G * sum of chunk partials + central term; per-body CM_acc terms.
__global__ void k_force_final(const double *__restrict__ part, int nch, long stride, Src s, int n,
                              const double *__restrict__ cm, double G, double M, int central, double *ax, double *ay,
                              double *az, double *cterm)
{
      int k = blockIdx.x * blockDim.x + threadIdx.x;
      if (k >= n) return;
      double a[3] = {0., 0., 0.};
      for (int c = 0; c < nch; c++)
            for (int d = 0; d < 3; d++) a[d] += part[(size_t)c * 3 * stride + d * stride + k];
      for (int d = 0; d < 3; d++) a[d] *= G;
      if (central) {
            double sx = s.x[k] - cm[0], sy = s.y[k] - cm[1], sz = s.z[k] - cm[2];
            double r2 = sx * sx + sy * sy + sz * sz;
            double ri = rsqrt(r2), i3 = ri * ri * ri;
            a[0] -= G * M * sx * i3; a[1] -= G * M * sy * i3; a[2] -= G * M * sz * i3;
            double g = G * s.m[k] * i3;
            cterm[k] = g * sx; cterm[n + k] = g * sy; cterm[2 * n + k] = g * sz;
      }
      ax[k] = a[0]; ay[k] = a[1]; az[k] = a[2];
}

// VJP outputs: mu (3), nu (1) per body; per-body terms of the CM-position VJP.
__global__ void k_vjp_final(const double *__restrict__ part, int nch, long stride, Src s, int n,
                            const double *__restrict__ cm, const double *__restrict__ Lam, double G, double M,
                            int central, double *mux, double *muy, double *muz, double *nu, double *xterm)
{
      int k = blockIdx.x * blockDim.x + threadIdx.x;
      if (k >= n) return;
      double o[4] = {0., 0., 0., 0.};
      for (int c = 0; c < nch; c++)
            for (int d = 0; d < 4; d++) o[d] += part[(size_t)c * 4 * stride + d * stride + k];
      for (int d = 0; d < 4; d++) o[d] *= G;
      if (central) {
            double sv[3] = {s.x[k] - cm[0], s.y[k] - cm[1], s.z[k] - cm[2]};
            double r2 = sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2];
            double ri = rsqrt(r2), i3 = ri * ri * ri, i5 = i3 * ri * ri;
            double mk = s.m[k];
            double lam[3] = {s.lx[k], s.ly[k], s.lz[k]};
            // w = m_k Lambda - M lambda_k ;  J w = w/|s|^3 - 3 s (s.w)/|s|^5
            double w[3], sw = 0.;
            for (int d = 0; d < 3; d++) { w[d] = mk * Lam[d] - M * lam[d]; sw += sv[d] * w[d]; }
            double Jw[3];
            for (int d = 0; d < 3; d++) Jw[d] = w[d] * i3 - 3.0 * sv[d] * sw * i5;
            for (int d = 0; d < 3; d++) {
                  o[d] += G * Jw[d];
                  xterm[d * n + k] = -G * Jw[d];  // G J (M lambda - m Lambda)
            }
            o[3] += G * (Lam[0] * sv[0] + Lam[1] * sv[1] + Lam[2] * sv[2]) * i3;
      }
      mux[k] = o[0]; muy[k] = o[1]; muz[k] = o[2]; nu[k] = o[3];
}

// JVP: d a = G * sum of chunk partials - G M J_k (dx_k - dX); per-body terms
// of d A_cm = sum_k G [dm_k s_k/|s|^3 + m_k J_k (dx_k - dX)].
__global__ void k_jvp_final(const double *__restrict__ part, int nch, long stride, Src s, int n,
                            const double *__restrict__ cm, const double *__restrict__ dX, double G, double M,
                            int central, double *dax, double *day, double *daz, double *cterm)
{
      int k = blockIdx.x * blockDim.x + threadIdx.x;
      if (k >= n) return;
      double o[3] = {0., 0., 0.};
      for (int c = 0; c < nch; c++)
            for (int d = 0; d < 3; d++) o[d] += part[(size_t)c * 3 * stride + d * stride + k];
      for (int d = 0; d < 3; d++) o[d] *= G;
      if (central) {
            double sv[3] = {s.x[k] - cm[0], s.y[k] - cm[1], s.z[k] - cm[2]};
            double r2 = sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2];
            double ri = rsqrt(r2), i3 = ri * ri * ri, i5 = i3 * ri * ri;
            double u[3] = {s.lx[k] - dX[0], s.ly[k] - dX[1], s.lz[k] - dX[2]};
            double su = sv[0] * u[0] + sv[1] * u[1] + sv[2] * u[2];
            double Ju[3];
            for (int d = 0; d < 3; d++) Ju[d] = u[d] * i3 - 3.0 * sv[d] * su * i5;
            const double mk = s.m[k], dmk = s.dm[k];
            for (int d = 0; d < 3; d++) {
                  o[d] -= G * M * Ju[d];
                  cterm[d * n + k] = G * (dmk * sv[d] * i3 + mk * Ju[d]);
            }
      }
      dax[k] = o[0]; day[k] = o[1]; daz[k] = o[2];
}

constexpr int SB = 256;
// out[d] = sum_k v[d*n + k], deterministic two levels (d < 3)
__global__ void k_sum3p(const double *__restrict__ v, int n, double *__restrict__ part)
{
      __shared__ double sh[3][SB];
      double a[3] = {0., 0., 0.};
      for (int k = blockIdx.x * SB + threadIdx.x; k < n; k += gridDim.x * SB)
            for (int d = 0; d < 3; d++) a[d] += v[(size_t)d * n + k];
      for (int d = 0; d < 3; d++) sh[d][threadIdx.x] = a[d];
      __syncthreads();
      for (int o = SB / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o)
                  for (int d = 0; d < 3; d++) sh[d][threadIdx.x] += sh[d][threadIdx.x + o];
            __syncthreads();
      }
      if (threadIdx.x < 3) part[blockIdx.x * 3 + threadIdx.x] = sh[threadIdx.x][0];
}

__global__ void k_sum3f(const double *__restrict__ part, int np, double *__restrict__ out)
{
      int d = threadIdx.x;
      if (d >= 3) return;
      double s = 0.;
      for (int b = 0; b < np; b++) s += part[3 * b + d];
      out[d] = s;
}

// y += a * x over 3 SoA blocks of n (and 3 CM components when cmy != nullptr)
__global__ void k_axpy3(double a, const double *__restrict__ x, double *__restrict__ y, int n, long stride,
                        const double *__restrict__ cmx, double *cmy)
{
      int k = blockIdx.x * blockDim.x + threadIdx.x;
      if (k < n)
            for (int d = 0; d < 3; d++) y[d * stride + k] += a * x[d * stride + k];
      if (k < 3 && cmy) cmy[k] += a * cmx[k];
}

__global__ void k_axpy1(double a, const double *__restrict__ x, double *__restrict__ y, int n)
{
      int k = blockIdx.x * blockDim.x + threadIdx.x;
      if (k < n) y[k] += a * x[k];
}

}  // namespace

namespace {

struct LF {
      int n, ntiles, tpc, nch, np;
      bool soft, central;
      double G, M;
      double *X, *V, *m, *sR, *cm, *acc, *cterm, *part, *red, *acm;
      double *lx, *lv, *LX, *LV, *mu, *nu, *gm, *xterm, *muX;
      double *ckpt, *seg;
      double *tx, *tv, *tm, *tX, *da, *dA;  // tangents (JVP)
      int C, ncp;
      cudaStream_t st;
};

int lf_force(LF &L, const double *pos, const double *cmpos)
{
      const int n = L.n;
      Src s{pos, pos + n, pos + 2 * n, L.m, L.sR, nullptr, nullptr, nullptr};
      dim3 grid(L.nch, L.ntiles);
      if (L.soft) k_pairs<0, true><<<grid, AT, 0, L.st>>>(s, n, L.tpc, L.part, n);
      else k_pairs<0, false><<<grid, AT, 0, L.st>>>(s, n, L.tpc, L.part, n);
      NCG_LAUNCHED();
      k_force_final<<<(n + 255) / 256, 256, 0, L.st>>>(L.part, L.nch, n, s, n, cmpos, L.G, L.M, L.central, L.acc,
                                                       L.acc + n, L.acc + 2 * n, L.cterm);
      NCG_LAUNCHED();
      if (L.central) {
            k_sum3p<<<L.np, SB, 0, L.st>>>(L.cterm, n, L.red);
            NCG_LAUNCHED();
            k_sum3f<<<1, 32, 0, L.st>>>(L.red, L.np, L.acm);
            NCG_LAUNCHED();
      }
      return NCGPU_OK;
}

// kick (v += dt a, CM too) then drift (x += dt v, CM too)
int lf_step(LF &L, double dt)
{
      NCG_TRY(lf_force(L, L.X, L.cm));
      const int n = L.n, nb = (n + 255) / 256;
      k_axpy3<<<nb, 256, 0, L.st>>>(dt, L.acc, L.V, n, n, L.acm, L.central ? L.cm + 3 : nullptr);
      NCG_LAUNCHED();
      k_axpy3<<<nb, 256, 0, L.st>>>(dt, L.V, L.X, n, n, L.cm + 3, L.central ? L.cm : nullptr);
      NCG_LAUNCHED();
      return NCGPU_OK;
}

int lf_vjp(LF &L, const double *pos, const double *cmpos)
{
      const int n = L.n;
      Src s{pos, pos + n, pos + 2 * n, L.m, L.sR, L.lv, L.lv + n, L.lv + 2 * n};
      dim3 grid(L.nch, L.ntiles);
      if (L.soft) k_pairs<1, true><<<grid, AT, 0, L.st>>>(s, n, L.tpc, L.part, n);
      else k_pairs<1, false><<<grid, AT, 0, L.st>>>(s, n, L.tpc, L.part, n);
      NCG_LAUNCHED();
      k_vjp_final<<<(n + 255) / 256, 256, 0, L.st>>>(L.part, L.nch, n, s, n, cmpos, L.LV, L.G, L.M, L.central, L.mu,
                                                     L.mu + n, L.mu + 2 * n, L.nu, L.xterm);
      NCG_LAUNCHED();
      if (L.central) {
            k_sum3p<<<L.np, SB, 0, L.st>>>(L.xterm, n, L.red);
            NCG_LAUNCHED();
            k_sum3f<<<1, 32, 0, L.st>>>(L.red, L.np, L.muX);
            NCG_LAUNCHED();
      }
      return NCGPU_OK;
}

// One kick + drift of the state and of its tangents.
int lf_step_jvp(LF &L, double dt)
{
      const int n = L.n, nb = (n + 255) / 256;
      NCG_TRY(lf_force(L, L.X, L.cm));
      Src s{L.X, L.X + n, L.X + 2 * n, L.m, L.sR, L.tx, L.tx + n, L.tx + 2 * n, L.tm};
      dim3 grid(L.nch, L.ntiles);
      if (L.soft) k_pairs<2, true><<<grid, AT, 0, L.st>>>(s, n, L.tpc, L.part, n);
      else k_pairs<2, false><<<grid, AT, 0, L.st>>>(s, n, L.tpc, L.part, n);
      NCG_LAUNCHED();
      k_jvp_final<<<nb, 256, 0, L.st>>>(L.part, L.nch, n, s, n, L.cm, L.tX, L.G, L.M, L.central, L.da, L.da + n,
                                        L.da + 2 * n, L.xterm);
      NCG_LAUNCHED();
      if (L.central) {
            k_sum3p<<<L.np, SB, 0, L.st>>>(L.xterm, n, L.red);
            NCG_LAUNCHED();
            k_sum3f<<<1, 32, 0, L.st>>>(L.red, L.np, L.dA);
            NCG_LAUNCHED();
      }
      k_axpy3<<<nb, 256, 0, L.st>>>(dt, L.acc, L.V, n, n, L.acm, L.central ? L.cm + 3 : nullptr);
      NCG_LAUNCHED();
      k_axpy3<<<nb, 256, 0, L.st>>>(dt, L.da, L.tv, n, n, L.dA, L.central ? L.tX + 3 : nullptr);
      NCG_LAUNCHED();
      k_axpy3<<<nb, 256, 0, L.st>>>(dt, L.V, L.X, n, n, L.cm + 3, L.central ? L.cm : nullptr);
      NCG_LAUNCHED();
      k_axpy3<<<nb, 256, 0, L.st>>>(dt, L.tv, L.tx, n, n, L.tX + 3, L.central ? L.tX : nullptr);
      NCG_LAUNCHED();
      return NCGPU_OK;
}

void split3(double *dst, const double *src, int n, cudaStream_t st, cudaError_t *e)
{
      for (int d = 0; d < 3 && *e == cudaSuccess; d++)
            *e = cudaMemcpy2DAsync(dst + (size_t)d * n, sizeof(double), src + d, 3 * sizeof(double), sizeof(double), n,
                                   cudaMemcpyHostToDevice, st);
}

void join3(double *dst, const double *src, int n, cudaStream_t st, cudaError_t *e)
{
      for (int d = 0; d < 3 && *e == cudaSuccess; d++)
            *e = cudaMemcpy2DAsync(dst + d, 3 * sizeof(double), src + (size_t)d * n, sizeof(double), sizeof(double), n,
                                   cudaMemcpyDeviceToHost, st);
}

// sR = sp * R, element by element (in place when sR == R)
__global__ void k_scale_R(const double *R, double sp, double *sR, int n)
{
      int k = blockIdx.x * blockDim.x + threadIdx.x;
      if (k < n) sR[k] = sp * R[k];
}

__global__ void k_xf(const double *__restrict__ X, const double *__restrict__ V, double h, double *__restrict__ out,
                     int n)
{
      int k = blockIdx.x * blockDim.x + threadIdx.x;
      if (k < n)
            for (int d = 0; d < 3; d++) out[(size_t)d * n + k] = X[(size_t)d * n + k] - h * V[(size_t)d * n + k];
}

int lf_run(const struct ncgpu_leapfrog_args *a, int mode)
{
      const bool vjp = mode == 1, jvp = mode == 2;
      Ctx &c = ctx();
      const int n = a->n;
      if (n <= 0 || !a->x0 || !a->v0 || !a->m || !a->R || !a->cm || a->nsteps < 0) return NCGPU_E_ARG;
      if (c.P.par_J2_bool) return NCGPU_E_UNSUPPORTED;  // the J2 term has no derivative kernels
      if (vjp && (!a->adj_x_final || !a->grad_x0 || !a->grad_v0 || !a->grad_m)) return NCGPU_E_ARG;
      if (jvp && (!a->tan_x0 || !a->tan_v0 || !a->tan_m || !a->tan_x_final)) return NCGPU_E_ARG;
      LF L{};
      L.n = n;
      L.st = c.s;
      L.G = c.P.par_G;
      L.M = a->cm[6];
      L.central = c.P.par_central_mass_bool != 0;
      L.soft = c.P.par_softening_parameter != 0.;
      L.ntiles = (n + AT - 1) / AT;
      L.nch = std::max(1, std::min(L.ntiles, (2048 + L.ntiles - 1) / L.ntiles));
      L.tpc = (L.ntiles + L.nch - 1) / L.nch;
      L.nch = (L.ntiles + L.tpc - 1) / L.tpc;
      L.np = std::min(128, (n + SB - 1) / SB);
      L.C = a->checkpoint > 0 ? a->checkpoint : 32;
      L.ncp = (a->nsteps + L.C - 1) / L.C + 1;
      const size_t N = (size_t)n, st = 6 * N + 6;
      size_t total = 3 * N * 2 + 2 * N + 6 + 3 * N + 3 * N + 4 * N * L.nch + 3 * 128 + 3  // X V m sR cm acc cterm part red acm
                     + 3 * N * 2 + 6 + 3 * N + N + N + 3 * N + 3                     // lx lv LX LV mu nu gm xterm muX
                     + st * L.ncp + (size_t)L.C * (3 * N + 3)                         // checkpoints, segment
                     + 3 * N * 3 + N + 6 + 3;                                         // tx tv tm tX da dA
      double *buf = nullptr;
      NCG_CK(cudaMalloc(&buf, total * sizeof(double)));
      double *p = buf;
      auto take = [&](size_t k) { double *q = p; p += k; return q; };
      L.X = take(3 * N); L.V = take(3 * N); L.m = take(N); L.sR = take(N); L.cm = take(6);
      L.acc = take(3 * N); L.cterm = take(3 * N); L.part = take(4 * N * L.nch); L.red = take(3 * 128);
      L.acm = take(3);
      L.lx = take(3 * N); L.lv = take(3 * N); L.LX = take(3); L.LV = take(3); L.mu = take(3 * N); L.nu = take(N);
      L.gm = take(N); L.xterm = take(3 * N); L.muX = take(3);
      L.ckpt = take(st * L.ncp); L.seg = take((size_t)L.C * (3 * N + 3));
      L.tx = take(3 * N); L.tv = take(3 * N); L.tm = take(N); L.tX = take(6); L.da = take(3 * N); L.dA = take(3);
      int status = NCGPU_OK;
      cudaError_t e = cudaSuccess;
      const double h = a->dt / 2.0, dt = a->dt;
      const int nb = (n + 255) / 256;
      split3(L.X, a->x0, n, L.st, &e);
      split3(L.V, a->v0, n, L.st, &e);
      if (e == cudaSuccess) e = cudaMemcpyAsync(L.m, a->m, sizeof(double) * N, cudaMemcpyHostToDevice, L.st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(L.sR, a->R, sizeof(double) * N, cudaMemcpyHostToDevice, L.st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(L.cm, a->cm, 6 * sizeof(double), cudaMemcpyHostToDevice, L.st);
      if (e == cudaSuccess) e = cudaMemsetAsync(L.acm, 0, 3 * sizeof(double), L.st);
      if (e != cudaSuccess) {
            cudaFree(buf);
            return cuda_fail(e, "leapfrog upload", __FILE__, __LINE__);
      }
#define LF_TRY(call)                         \
      do {                                   \
            if ((status = (call)) != NCGPU_OK) goto done; \
      } while (0)
#define LF_LAUNCHED()                                                                 \
      do {                                                                            \
            note_launch();                                                            \
            cudaError_t e_ = cudaGetLastError();                                      \
            if (e_ != cudaSuccess) { status = cuda_fail(e_, "launch", __FILE__, __LINE__); goto done; } \
      } while (0)
      k_scale_R<<<nb, 256, 0, L.st>>>(L.sR, c.P.par_softening_parameter, L.sR, n);
      LF_LAUNCHED();
      if (jvp) {
            split3(L.tx, a->tan_x0, n, L.st, &e);
            split3(L.tv, a->tan_v0, n, L.st, &e);
            if (e == cudaSuccess) e = cudaMemcpyAsync(L.tm, a->tan_m, sizeof(double) * N, cudaMemcpyHostToDevice, L.st);
            if (e == cudaSuccess) e = cudaMemsetAsync(L.tX, 0, 6 * sizeof(double), L.st);
            if (e != cudaSuccess) { status = cuda_fail(e, "tangent upload", __FILE__, __LINE__); goto done; }
            k_axpy3<<<nb, 256, 0, L.st>>>(h, L.tv, L.tx, n, n, nullptr, nullptr);
            LF_LAUNCHED();
      }
      // half drift (src/rk4.c:873-880)
      k_axpy3<<<nb, 256, 0, L.st>>>(h, L.V, L.X, n, n, L.cm + 3, L.central ? L.cm : nullptr);
      LF_LAUNCHED();
      for (int s = 0; s < a->nsteps; s++) {
            if (vjp && s % L.C == 0) {
                  double *ck = L.ckpt + st * (s / L.C);
                  e = cudaMemcpyAsync(ck, L.X, sizeof(double) * 6 * N, cudaMemcpyDeviceToDevice, L.st);
                  if (e == cudaSuccess) e = cudaMemcpyAsync(ck + 6 * N, L.cm, 6 * sizeof(double), cudaMemcpyDeviceToDevice, L.st);
                  if (e != cudaSuccess) { status = cuda_fail(e, "checkpoint", __FILE__, __LINE__); goto done; }
            }
            if (jvp) LF_TRY(lf_step_jvp(L, dt));
            else LF_TRY(lf_step(L, dt));
      }
      if (jvp) {
            k_xf<<<nb, 256, 0, L.st>>>(L.tx, L.tv, h, L.da, n);
            LF_LAUNCHED();
            join3(a->tan_x_final, L.da, n, L.st, &e);
            if (e == cudaSuccess) e = cudaStreamSynchronize(L.st);
            if (e != cudaSuccess) { status = cuda_fail(e, "tangent download", __FILE__, __LINE__); goto done; }
      }
      if (a->x_final || a->v_final) {
            k_xf<<<nb, 256, 0, L.st>>>(L.X, L.V, h, L.acc, n);  // half back-drift of the output (src/rk4.c:929-936)
            LF_LAUNCHED();
            if (a->x_final) join3(a->x_final, L.acc, n, L.st, &e);
            if (a->v_final) join3(a->v_final, L.V, n, L.st, &e);
            if (e == cudaSuccess) e = cudaStreamSynchronize(L.st);
            if (e != cudaSuccess) { status = cuda_fail(e, "leapfrog download", __FILE__, __LINE__); goto done; }
      }
      if (vjp) {
            // x_F = x_n - h v_n
            split3(L.lx, a->adj_x_final, n, L.st, &e);
            if (e == cudaSuccess) e = cudaMemsetAsync(L.lv, 0, sizeof(double) * 3 * N, L.st);
            if (e == cudaSuccess) e = cudaMemsetAsync(L.LX, 0, 6 * sizeof(double), L.st);  // LX, LV
            if (e == cudaSuccess) e = cudaMemsetAsync(L.gm, 0, sizeof(double) * N, L.st);
            if (e != cudaSuccess) { status = cuda_fail(e, "adjoint init", __FILE__, __LINE__); goto done; }
            k_axpy3<<<nb, 256, 0, L.st>>>(-h, L.lx, L.lv, n, n, nullptr, nullptr);
            LF_LAUNCHED();
            for (int q = (a->nsteps - 1) / L.C; q >= 0 && a->nsteps > 0; q--) {
                  const int s0 = q * L.C, s1 = std::min(a->nsteps, s0 + L.C);
                  const double *ck = L.ckpt + st * q;
                  e = cudaMemcpyAsync(L.X, ck, sizeof(double) * 6 * N, cudaMemcpyDeviceToDevice, L.st);
                  if (e == cudaSuccess) e = cudaMemcpyAsync(L.cm, ck + 6 * N, 6 * sizeof(double), cudaMemcpyDeviceToDevice, L.st);
                  if (e != cudaSuccess) { status = cuda_fail(e, "restore", __FILE__, __LINE__); goto done; }
                  for (int s = s0; s < s1; s++) {  // recompute, keeping the positions each kick saw
                        double *sg = L.seg + (size_t)(s - s0) * (3 * N + 3);
                        e = cudaMemcpyAsync(sg, L.X, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, L.st);
                        if (e == cudaSuccess) e = cudaMemcpyAsync(sg + 3 * N, L.cm, 3 * sizeof(double), cudaMemcpyDeviceToDevice, L.st);
                        if (e != cudaSuccess) { status = cuda_fail(e, "segment", __FILE__, __LINE__); goto done; }
                        LF_TRY(lf_step(L, dt));
                  }
                  for (int s = s1 - 1; s >= s0; s--) {
                        const double *sg = L.seg + (size_t)(s - s0) * (3 * N + 3);
                        // drift x_{s+1} = x_s + dt v_{s+1}
                        k_axpy3<<<nb, 256, 0, L.st>>>(dt, L.lx, L.lv, n, n, L.LX, L.LV);
                        LF_LAUNCHED();
                        // kick v_{s+1} = v_s + dt a(x_s)
                        LF_TRY(lf_vjp(L, sg, sg + 3 * N));
                        k_axpy3<<<nb, 256, 0, L.st>>>(dt, L.mu, L.lx, n, n, L.muX, L.central ? L.LX : nullptr);
                        LF_LAUNCHED();
                        k_axpy1<<<nb, 256, 0, L.st>>>(dt, L.nu, L.gm, n);
                        LF_LAUNCHED();
                  }
            }
            // initial half drift x = x0 + h v0
            k_axpy3<<<nb, 256, 0, L.st>>>(h, L.lx, L.lv, n, n, nullptr, nullptr);
            LF_LAUNCHED();
            join3(a->grad_x0, L.lx, n, L.st, &e);
            join3(a->grad_v0, L.lv, n, L.st, &e);
            if (e == cudaSuccess) e = cudaMemcpyAsync(a->grad_m, L.gm, sizeof(double) * N, cudaMemcpyDeviceToHost, L.st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(L.st);
            if (e != cudaSuccess) { status = cuda_fail(e, "adjoint download", __FILE__, __LINE__); goto done; }
      }
#undef LF_TRY
#undef LF_LAUNCHED
done:
      cudaStreamSynchronize(L.st);
      cudaFree(buf);
      return status;
}

}  // namespace
}  // namespace ncg

using namespace ncg;

extern "C" int ncgpu_leapfrog(const struct ncgpu_leapfrog_args *args)
{
      reset_launches();
      if (!ctx().inited) return NCGPU_E_STATE;
      if (!args) return NCGPU_E_ARG;
      return lf_run(args, 0);
}

extern "C" int ncgpu_leapfrog_vjp(const struct ncgpu_leapfrog_args *args)
{
      reset_launches();
      if (!ctx().inited) return NCGPU_E_STATE;
      if (!args) return NCGPU_E_ARG;
      return lf_run(args, 1);
}

extern "C" int ncgpu_leapfrog_jvp(const struct ncgpu_leapfrog_args *args)
{
      reset_launches();
      if (!ctx().inited) return NCGPU_E_STATE;
      if (!args) return NCGPU_E_ARG;
      return lf_run(args, 2);
}
