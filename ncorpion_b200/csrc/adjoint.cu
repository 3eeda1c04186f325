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
// (target block, source chunk) work units reduced in a fixed order.  In the
// MIXED gravity mode the bodies are taken in the Morton order of their initial
// positions (a permutation done on the host at the call's boundary), every
// evaluation computes the 128-body tiles' boxes, and only the tile pairs whose
// boxes are near (near_theta x the larger diagonal, and each tile with itself)
// are summed in FP64; the others in FP32 on coordinates relative to the source
// tile's centre, the FP32 sums of every 64 sources folded into FP64 -- the
// force kernel's scheme applied to the force, its VJP and its JVP.
#include <algorithm>
#include <vector>
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

// One warp per tile: centre and half extents of its bodies' box.
__global__ void k_adj_tilebox(const double *__restrict__ pos, int n, int ntiles, double *__restrict__ box)
{
      const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
      if (warp >= ntiles) return;
      const int base = warp * AT, cnt = min(AT, n - base);
      double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
      for (int j = lane; j < cnt; j += 32)
            for (int d = 0; d < 3; d++) {
                  const double v = pos[(size_t)d * n + base + j];
                  lo[d] = fmin(lo[d], v);
                  hi[d] = fmax(hi[d], v);
            }
      for (int o = 16; o > 0; o >>= 1)
            for (int d = 0; d < 3; d++) {
                  lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
                  hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
            }
      if (lane < 3) {
            box[warp * 6 + lane] = 0.5 * (lo[lane] + hi[lane]);
            box[warp * 6 + 3 + lane] = 0.5 * (hi[lane] - lo[lane]);
      }
}

// k_pairs in the MIXED mode: FP64 for near tile pairs (the same pair terms),
// FP32 relative to the source tile's centre for the others, with packed f32x2
// arithmetic (two sources per instruction) for the force and its VJP.  (Two
// targets a thread measured slower: 1.56 against 1.15 ms per forward+adjoint
// step at N = 16,384, from 128 registers a thread and the serial FP64 near
// tiles.)
template <int OP, bool SOFT>
__global__ void __launch_bounds__(AT) k_pairs_mx(Src s, int n, int tpc, const double *__restrict__ box, double theta,
                                                 double *__restrict__ part, long stride)
{
      __shared__ double sx[AT], sy[AT], sz[AT], sm[AT], sr[AT], slx[AT], sly[AT], slz[AT], sdm[AT];
      __shared__ __align__(16) float fx[AT], fy[AT], fz[AT], fm[AT], fr[AT], flx[AT], fly[AT], flz[AT], fdm[AT];
      const int ib = blockIdx.y;
      const int k = ib * AT + threadIdx.x;
      const bool act = k < n;
      const int kk = act ? k : 0;
      const double xk = s.x[kk], yk = s.y[kk], zk = s.z[kk], mk = s.m[kk], rk = SOFT ? s.sR[kk] : 0.;
      double lxk = 0., lyk = 0., lzk = 0.;
      if (OP >= 1) { lxk = s.lx[kk]; lyk = s.ly[kk]; lzk = s.lz[kk]; }
      const float mkf = (float)mk, rkf = (float)rk, lxkf = (float)lxk, lykf = (float)lyk, lzkf = (float)lzk;
      double o0 = 0., o1 = 0., o2 = 0., o3 = 0.;
      const int ntiles = (n + AT - 1) / AT;
      const int t0 = blockIdx.x * tpc, t1 = min(ntiles, t0 + tpc);
      const double *bi = box + 6 * ib;
      for (int t = t0; t < t1; ++t) {
            const int j = t * AT + threadIdx.x;
            const double *bj = box + 6 * t;
            const bool near = t == ib || tiles_near(bi, bj, theta);
            __syncthreads();
            if (j >= n && !near) {  // padding of the far path: far away, massless, no adjoint
                  fx[threadIdx.x] = fy[threadIdx.x] = fz[threadIdx.x] = 1e18f;
                  fm[threadIdx.x] = fr[threadIdx.x] = flx[threadIdx.x] = fly[threadIdx.x] = flz[threadIdx.x] = 0.f;
                  fdm[threadIdx.x] = 0.f;
            }
            if (j < n) {
                  if (near) {
                        sx[threadIdx.x] = s.x[j]; sy[threadIdx.x] = s.y[j]; sz[threadIdx.x] = s.z[j];
                        sm[threadIdx.x] = s.m[j];
                        if (SOFT) sr[threadIdx.x] = s.sR[j];
                        if (OP >= 1) { slx[threadIdx.x] = s.lx[j]; sly[threadIdx.x] = s.ly[j]; slz[threadIdx.x] = s.lz[j]; }
                        if (OP == 2) sdm[threadIdx.x] = s.dm[j];
                  } else {
                        fx[threadIdx.x] = (float)(s.x[j] - bj[0]);
                        fy[threadIdx.x] = (float)(s.y[j] - bj[1]);
                        fz[threadIdx.x] = (float)(s.z[j] - bj[2]);
                        fm[threadIdx.x] = (float)s.m[j];
                        if (SOFT) fr[threadIdx.x] = (float)s.sR[j];
                        if (OP >= 1) {
                              flx[threadIdx.x] = (float)s.lx[j]; fly[threadIdx.x] = (float)s.ly[j];
                              flz[threadIdx.x] = (float)s.lz[j];
                        }
                        if (OP == 2) fdm[threadIdx.x] = (float)s.dm[j];
                  }
            }
            __syncthreads();
            const int cnt = min(AT, n - t * AT);
            if (near) {
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
            } else if (OP == 0) {
                  // packed f32x2: two sources per instruction; FP32 runs of 64 sources
                  const float xr = (float)(xk - bj[0]), yr = (float)(yk - bj[1]), zr = (float)(zk - bj[2]);
                  const f2 XT = f2_pack(xr, xr), YT = f2_pack(yr, yr), ZT = f2_pack(zr, zr), RT = f2_pack(rkf, rkf);
                  const int ce = (cnt + 1) & ~1;
                  for (int q0 = 0; q0 < ce; q0 += 64) {
                        f2 P0 = 0ull, P1 = 0ull, P2 = 0ull;
                        const int qe = min(ce, q0 + 64);
#pragma unroll 4
                        for (int q = q0; q < qe; q += 2) {
                              const f2 dx = f2_sub(*(const f2 *)&fx[q], XT), dy = f2_sub(*(const f2 *)&fy[q], YT);
                              const f2 dz = f2_sub(*(const f2 *)&fz[q], ZT);
                              f2 d2;
                              if (SOFT) {
                                    const f2 e = f2_add(*(const f2 *)&fr[q], RT);
                                    d2 = f2_fma(dx, dx, f2_mul(e, e));
                              } else {
                                    d2 = f2_mul(dx, dx);
                              }
                              d2 = f2_fma(dy, dy, d2);
                              d2 = f2_fma(dz, dz, d2);
                              const f2 i = f2_rsqrt(d2);
                              const f2 w = f2_mul(f2_mul(*(const f2 *)&fm[q], i), f2_mul(i, i));
                              P0 = f2_fma(w, dx, P0);
                              P1 = f2_fma(w, dy, P1);
                              P2 = f2_fma(w, dz, P2);
                        }
                        float lo, hi;
                        f2_unpack(P0, lo, hi); o0 += (double)lo + (double)hi;
                        f2_unpack(P1, lo, hi); o1 += (double)lo + (double)hi;
                        f2_unpack(P2, lo, hi); o2 += (double)lo + (double)hi;
                  }
            } else if (OP == 1) {
                  // the VJP's pair terms, packed as OP 0
                  const float xr = (float)(xk - bj[0]), yr = (float)(yk - bj[1]), zr = (float)(zk - bj[2]);
                  const f2 XT = f2_pack(xr, xr), YT = f2_pack(yr, yr), ZT = f2_pack(zr, zr), RT = f2_pack(rkf, rkf);
                  const f2 MK = f2_pack(mkf, mkf), NLX = f2_pack(-lxkf, -lxkf), NLY = f2_pack(-lykf, -lykf),
                           NLZ = f2_pack(-lzkf, -lzkf), NEG3 = f2_pack(-3.f, -3.f);
                  // sources q, q + 1 packed, four per 128-bit shared load (a far tile is
                  // padded with far, massless sources up to a multiple of four)
                  const int ce = (cnt + 3) & ~3;
                  for (int q0 = 0; q0 < ce; q0 += 64) {
                        f2 P0 = 0ull, P1 = 0ull, P2 = 0ull, P3 = 0ull;
                        const int qe = min(ce, q0 + 64);
                        auto term = [&](f2 XS, f2 YS, f2 ZS, f2 RS, f2 mj, f2 LX, f2 LY, f2 LZ) {
                              const f2 rx = f2_sub(XS, XT), ry = f2_sub(YS, YT), rz = f2_sub(ZS, ZT);
                              f2 d2;
                              if (SOFT) {
                                    const f2 e = f2_add(RS, RT);
                                    d2 = f2_fma(rx, rx, f2_mul(e, e));
                              } else {
                                    d2 = f2_mul(rx, rx);
                              }
                              d2 = f2_fma(ry, ry, d2);
                              d2 = f2_fma(rz, rz, d2);
                              const f2 ri = f2_rsqrt(d2);
                              const f2 r2i = f2_mul(ri, ri);
                              const f2 i3 = f2_mul(r2i, ri), i5 = f2_mul(i3, r2i);
                              // w = m_k lambda_j - m_j lambda_k
                              const f2 wx = f2_fma(mj, NLX, f2_mul(MK, LX)), wy = f2_fma(mj, NLY, f2_mul(MK, LY));
                              const f2 wz = f2_fma(mj, NLZ, f2_mul(MK, LZ));
                              const f2 rw = f2_fma(rz, wz, f2_fma(ry, wy, f2_mul(rx, wx)));
                              const f2 nc = f2_mul(f2_mul(NEG3, rw), i5);  // -3 (r . w) / D^5
                              P0 = f2_fma(wx, i3, f2_fma(rx, nc, P0));
                              P1 = f2_fma(wy, i3, f2_fma(ry, nc, P1));
                              P2 = f2_fma(wz, i3, f2_fma(rz, nc, P2));
                              const f2 lr = f2_fma(LZ, rz, f2_fma(LY, ry, f2_mul(LX, rx)));
                              P3 = f2_sub(P3, f2_mul(lr, i3));
                        };
#pragma unroll 1
                        for (int q = q0; q < qe; q += 4) {
                              const ulonglong2 X = *(const ulonglong2 *)&fx[q], Y = *(const ulonglong2 *)&fy[q];
                              const ulonglong2 Z = *(const ulonglong2 *)&fz[q], M = *(const ulonglong2 *)&fm[q];
                              const ulonglong2 LX = *(const ulonglong2 *)&flx[q], LY = *(const ulonglong2 *)&fly[q];
                              const ulonglong2 LZ = *(const ulonglong2 *)&flz[q];
                              ulonglong2 R = make_ulonglong2(0ull, 0ull);
                              if (SOFT) R = *(const ulonglong2 *)&fr[q];
                              term(X.x, Y.x, Z.x, R.x, M.x, LX.x, LY.x, LZ.x);
                              term(X.y, Y.y, Z.y, R.y, M.y, LX.y, LY.y, LZ.y);
                        }
                        float lo, hi;
                        f2_unpack(P0, lo, hi); o0 += (double)lo + (double)hi;
                        f2_unpack(P1, lo, hi); o1 += (double)lo + (double)hi;
                        f2_unpack(P2, lo, hi); o2 += (double)lo + (double)hi;
                        f2_unpack(P3, lo, hi); o3 += (double)lo + (double)hi;
                  }
            } else {  // OP 2 (the JVP), scalar FP32
                  const float xr = (float)(xk - bj[0]), yr = (float)(yk - bj[1]), zr = (float)(zk - bj[2]);
                  for (int q0 = 0; q0 < cnt; q0 += 64) {  // FP32 runs of 64 sources
                        float p0 = 0.f, p1 = 0.f, p2 = 0.f;
                        const int qe = min(cnt, q0 + 64);
                        for (int q = q0; q < qe; ++q) {
                              const float rx = fx[q] - xr, ry = fy[q] - yr, rz = fz[q] - zr;
                              float d2 = 0.f;
                              if (SOFT) { const float e = rkf + fr[q]; d2 = e * e; }
                              d2 = fmaf(rx, rx, fmaf(ry, ry, fmaf(rz, rz, d2)));
                              const float ri = rsqrtf(d2);
                              const float i3 = ri * ri * ri, i5 = i3 * ri * ri;
                              const float dx = flx[q] - lxkf, dy = fly[q] - lykf, dz = flz[q] - lzkf;
                              const float rd = rx * dx + ry * dy + rz * dz;
                              const float mj = fm[q], c = 3.f * rd * i5 * mj, g = fdm[q] * i3;
                              p0 += g * rx + mj * i3 * dx - rx * c;
                              p1 += g * ry + mj * i3 * dy - ry * c;
                              p2 += g * rz + mj * i3 * dz - rz * c;
                        }
                        o0 += (double)p0; o1 += (double)p1; o2 += (double)p2;
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
constexpr int SB = 256;  // threads of the fold kernels and of the two-level sums

// The block's sums of three per-body terms (zero past n): part[3 b + d] for
// block b; k_sum3f then adds the blocks' sums in block order (deterministic).
__device__ __forceinline__ void block_sum3(double v0, double v1, double v2, double *__restrict__ part)
{
      __shared__ double sh[3][SB];
      sh[0][threadIdx.x] = v0;
      sh[1][threadIdx.x] = v1;
      sh[2][threadIdx.x] = v2;
      __syncthreads();
      for (int o = SB / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o)
                  for (int d = 0; d < 3; d++) sh[d][threadIdx.x] += sh[d][threadIdx.x + o];
            __syncthreads();
      }
      if (threadIdx.x < 3) part[blockIdx.x * 3 + threadIdx.x] = sh[threadIdx.x][0];
}


// acc = G * sum of chunk partials + central term; per-body CM_acc terms.
__global__ void __launch_bounds__(SB) k_force_final(const double *__restrict__ part, int nch, long stride, Src s,
                                                    int n, const double *__restrict__ cm, double G, double M,
                                                    int central, double *ax, double *ay, double *az,
                                                    double *__restrict__ red)
{
      const int k = blockIdx.x * blockDim.x + threadIdx.x;
      double c[3] = {0., 0., 0.};
      if (k < n) {
            double a[3] = {0., 0., 0.};
#pragma unroll 8  // the chunks' loads in flight together (sums still in chunk order)
            for (int ch = 0; ch < nch; ch++)
                  for (int d = 0; d < 3; d++) a[d] += part[(size_t)ch * 3 * stride + d * stride + k];
            for (int d = 0; d < 3; d++) a[d] *= G;
            if (central) {
                  double sx = s.x[k] - cm[0], sy = s.y[k] - cm[1], sz = s.z[k] - cm[2];
                  double r2 = sx * sx + sy * sy + sz * sz;
                  double ri = rsqrt(r2), i3 = ri * ri * ri;
                  a[0] -= G * M * sx * i3; a[1] -= G * M * sy * i3; a[2] -= G * M * sz * i3;
                  double g = G * s.m[k] * i3;
                  c[0] = g * sx; c[1] = g * sy; c[2] = g * sz;
            }
            ax[k] = a[0]; ay[k] = a[1]; az[k] = a[2];
      }
      if (central) block_sum3(c[0], c[1], c[2], red);  // the CM_acc terms (central is uniform)
}

// VJP outputs: mu (3), nu (1) per body; per-body terms of the CM-position VJP.
__global__ void __launch_bounds__(SB) k_vjp_final(const double *__restrict__ part, int nch, long stride, Src s,
                                                  int n, const double *__restrict__ cm,
                                                  const double *__restrict__ Lam, double G, double M, int central,
                                                  double *mux, double *muy, double *muz, double *nu,
                                                  double *__restrict__ red)
{
      const int k = blockIdx.x * blockDim.x + threadIdx.x;
      double xt[3] = {0., 0., 0.};
      if (k < n) {
      double o[4] = {0., 0., 0., 0.};
#pragma unroll 8  // the chunks' loads in flight together (sums still in chunk order)
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
                  xt[d] = -G * Jw[d];  // G J (M lambda - m Lambda)
            }
            o[3] += G * (Lam[0] * sv[0] + Lam[1] * sv[1] + Lam[2] * sv[2]) * i3;
      }
      mux[k] = o[0]; muy[k] = o[1]; muz[k] = o[2]; nu[k] = o[3];
      }
      if (central) block_sum3(xt[0], xt[1], xt[2], red);  // the CM-position VJP's terms
}

// JVP: d a = G * sum of chunk partials - G M J_k (dx_k - dX); per-body terms
// of d A_cm = sum_k G [dm_k s_k/|s|^3 + m_k J_k (dx_k - dX)].
__global__ void __launch_bounds__(SB) k_jvp_final(const double *__restrict__ part, int nch, long stride, Src s,
                                                  int n, const double *__restrict__ cm,
                                                  const double *__restrict__ dX, double G, double M, int central,
                                                  double *dax, double *day, double *daz, double *__restrict__ red)
{
      const int k = blockIdx.x * blockDim.x + threadIdx.x;
      double ct[3] = {0., 0., 0.};
      if (k < n) {
      double o[3] = {0., 0., 0.};
#pragma unroll 8  // the chunks' loads in flight together (sums still in chunk order)
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
                  ct[d] = G * (dmk * sv[d] * i3 + mk * Ju[d]);
            }
      }
      dax[k] = o[0]; day[k] = o[1]; daz[k] = o[2];
      }
      if (central) block_sum3(ct[0], ct[1], ct[2], red);  // the terms of d A_cm
}

// out[d] = the sum of the blocks' partial sums part[3 b + d] (block_sum3), in
// block order (d < 3)
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
      double *X, *V, *m, *sR, *cm, *acc, *part, *red, *acm;
      double *lx, *lv, *LX, *LV, *mu, *nu, *gm, *muX;
      double *ckpt, *seg;
      double *tx, *tv, *tm, *tX, *da, *dA;  // tangents (JVP)
      int C, ncp;
      bool mixed;                  // MIXED gravity mode: k_pairs_mx with tile boxes
      double theta, *box;
      double *boxseg;              // mixed mode: the tile boxes of a segment's recomputed steps
      cudaStream_t st;
};

// the pair sums of OP over positions pos; the mixed mode's tile boxes in box
// (null: L.box), computed from pos first unless `have_box`
template <int OP>
int lf_pairs(LF &L, const Src &s, const double *pos, double *box = nullptr, bool have_box = false)
{
      const int n = L.n;
      dim3 grid(L.nch, L.ntiles);
      if (L.mixed) {
            if (!box) box = L.box;
            if (!have_box) {
                  k_adj_tilebox<<<(L.ntiles * 32 + 255) / 256, 256, 0, L.st>>>(pos, n, L.ntiles, box);
                  NCG_LAUNCHED();
            }
            if (L.soft) k_pairs_mx<OP, true><<<grid, AT, 0, L.st>>>(s, n, L.tpc, box, L.theta, L.part, n);
            else k_pairs_mx<OP, false><<<grid, AT, 0, L.st>>>(s, n, L.tpc, box, L.theta, L.part, n);
      } else {
            if (L.soft) k_pairs<OP, true><<<grid, AT, 0, L.st>>>(s, n, L.tpc, L.part, n);
            else k_pairs<OP, false><<<grid, AT, 0, L.st>>>(s, n, L.tpc, L.part, n);
      }
      NCG_LAUNCHED();
      return NCGPU_OK;
}

int lf_force(LF &L, const double *pos, const double *cmpos, double *box = nullptr)
{
      const int n = L.n;
      Src s{pos, pos + n, pos + 2 * n, L.m, L.sR, nullptr, nullptr, nullptr};
      NCG_TRY(lf_pairs<0>(L, s, pos, box));
      const int nb = (n + SB - 1) / SB;
      k_force_final<<<nb, SB, 0, L.st>>>(L.part, L.nch, n, s, n, cmpos, L.G, L.M, L.central, L.acc, L.acc + n,
                                         L.acc + 2 * n, L.red);
      NCG_LAUNCHED();
      if (L.central) {
            k_sum3f<<<1, 32, 0, L.st>>>(L.red, nb, L.acm);
            NCG_LAUNCHED();
      }
      return NCGPU_OK;
}

// kick (v += dt a, CM too) then drift (x += dt v, CM too); box: where the
// force's tile boxes go (null: L.box)
int lf_step(LF &L, double dt, double *box = nullptr)
{
      NCG_TRY(lf_force(L, L.X, L.cm, box));
      const int n = L.n, nb = (n + 255) / 256;
      k_axpy3<<<nb, 256, 0, L.st>>>(dt, L.acc, L.V, n, n, L.acm, L.central ? L.cm + 3 : nullptr);
      NCG_LAUNCHED();
      k_axpy3<<<nb, 256, 0, L.st>>>(dt, L.V, L.X, n, n, L.cm + 3, L.central ? L.cm : nullptr);
      NCG_LAUNCHED();
      return NCGPU_OK;
}

// box: the tile boxes of pos when known (null: computed)
int lf_vjp(LF &L, const double *pos, const double *cmpos, double *box = nullptr)
{
      const int n = L.n;
      Src s{pos, pos + n, pos + 2 * n, L.m, L.sR, L.lv, L.lv + n, L.lv + 2 * n};
      NCG_TRY(lf_pairs<1>(L, s, pos, box, box != nullptr));
      const int nb = (n + SB - 1) / SB;
      k_vjp_final<<<nb, SB, 0, L.st>>>(L.part, L.nch, n, s, n, cmpos, L.LV, L.G, L.M, L.central, L.mu, L.mu + n,
                                       L.mu + 2 * n, L.nu, L.red);
      NCG_LAUNCHED();
      if (L.central) {
            k_sum3f<<<1, 32, 0, L.st>>>(L.red, nb, L.muX);
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
      NCG_TRY(lf_pairs<2>(L, s, L.X));
      const int nbs = (n + SB - 1) / SB;
      k_jvp_final<<<nbs, SB, 0, L.st>>>(L.part, L.nch, n, s, n, L.cm, L.tX, L.G, L.M, L.central, L.da, L.da + n,
                                        L.da + 2 * n, L.red);
      NCG_LAUNCHED();
      if (L.central) {
            k_sum3f<<<1, 32, 0, L.st>>>(L.red, nbs, L.dA);
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

int lf_core(const struct ncgpu_leapfrog_args *a, int mode, bool mixed)
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
      if (mixed) {
            // (target tile, source chunk) work units: about 8 per resident CTA
            // slot, so that the last wave is short
            int occ = 1;
            NCG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pairs_mx<1, true>, AT, 0));
            const long want = 8L * std::max(occ, 1) * c.sm_count;
            L.nch = (int)std::max(1L, std::min((long)L.ntiles, (want + L.ntiles - 1) / L.ntiles));
      } else {
            L.nch = std::max(1, std::min(L.ntiles, (2048 + L.ntiles - 1) / L.ntiles));
      }
      L.tpc = (L.ntiles + L.nch - 1) / L.nch;
      L.nch = (L.ntiles + L.tpc - 1) / L.tpc;
      L.np = (n + SB - 1) / SB;  // blocks of the fold kernels: their CM sums in red
      L.mixed = mixed;
      L.theta = c.P.par_near_theta > 0. ? c.P.par_near_theta : 0.15;
      L.C = a->checkpoint > 0 ? a->checkpoint : 32;
      L.ncp = (a->nsteps + L.C - 1) / L.C + 1;
      const size_t N = (size_t)n, st = 6 * N + 6;
      size_t total = 3 * N * 2 + 2 * N + 6 + 3 * N + 4 * N * L.nch + 3 * (size_t)L.np + 3  // X V m sR cm acc part red acm
                     + 3 * N * 2 + 6 + 3 * N + N + N + 3                              // lx lv LX LV mu nu gm muX
                     + st * L.ncp + (size_t)L.C * (3 * N + 3)                         // checkpoints, segment
                     + 3 * N * 3 + N + 6 + 3                                          // tx tv tm tX da dA
                     + 6 * (size_t)L.ntiles                                           // tile boxes
                     + (mixed && vjp ? 6 * (size_t)L.ntiles * L.C : 0);               // a segment's boxes
      if (total > c.lf_cap) {  // grown when needed, kept for the next call
            if (c.lf_buf) cudaFree(c.lf_buf);
            c.lf_buf = nullptr;
            c.lf_cap = 0;
            NCG_CK(cudaMalloc(&c.lf_buf, total * sizeof(double)));
            c.lf_cap = total;
      }
      double *p = c.lf_buf;
      auto take = [&](size_t k) { double *q = p; p += k; return q; };
      L.X = take(3 * N); L.V = take(3 * N); L.m = take(N); L.sR = take(N); L.cm = take(6);
      L.acc = take(3 * N); L.part = take(4 * N * L.nch); L.red = take(3 * (size_t)L.np);
      L.acm = take(3);
      L.lx = take(3 * N); L.lv = take(3 * N); L.LX = take(3); L.LV = take(3); L.mu = take(3 * N); L.nu = take(N);
      L.gm = take(N); L.muX = take(3);
      L.ckpt = take(st * L.ncp); L.seg = take((size_t)L.C * (3 * N + 3));
      L.tx = take(3 * N); L.tv = take(3 * N); L.tm = take(N); L.tX = take(6); L.da = take(3 * N); L.dA = take(3);
      L.box = take(6 * (size_t)L.ntiles);
      L.boxseg = take(mixed && vjp ? 6 * (size_t)L.ntiles * L.C : 0);
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
      if (e != cudaSuccess) return cuda_fail(e, "leapfrog upload", __FILE__, __LINE__);
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
                        LF_TRY(lf_step(L, dt, L.mixed ? L.boxseg + (size_t)(s - s0) * 6 * L.ntiles : nullptr));
                  }
                  for (int s = s1 - 1; s >= s0; s--) {
                        const double *sg = L.seg + (size_t)(s - s0) * (3 * N + 3);
                        // drift x_{s+1} = x_s + dt v_{s+1}
                        k_axpy3<<<nb, 256, 0, L.st>>>(dt, L.lx, L.lv, n, n, L.LX, L.LV);
                        LF_LAUNCHED();
                        // kick v_{s+1} = v_s + dt a(x_s)
                        // (the recomputation's boxes of these positions)
                        LF_TRY(lf_vjp(L, sg, sg + 3 * N, L.mixed ? L.boxseg + (size_t)(s - s0) * 6 * L.ntiles : nullptr));
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
      return status;
}

// Morton order (30-bit keys from one cubic quantisation of the bounding box)
// of n positions given as 3n AoS doubles: perm[i] = the body at position i.
void morton_order(const double *x, int n, std::vector<int> &perm)
{
      double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
      for (int k = 0; k < n; k++)
            for (int d = 0; d < 3; d++) {
                  lo[d] = std::min(lo[d], x[3 * k + d]);
                  hi[d] = std::max(hi[d], x[3 * k + d]);
            }
      const double ext = std::max(std::max(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]);
      std::vector<uint32_t> key(n);
      for (int k = 0; k < n; k++) {
            uint32_t q[3];
            for (int d = 0; d < 3; d++) {
                  const double f = ext > 0. ? (x[3 * k + d] - lo[d]) / ext : 0.;
                  q[d] = (uint32_t)std::min(std::max((int)(f * 1023.999), 0), 1023);
            }
            uint32_t m = 0;
            for (int b = 9; b >= 0; b--)
                  for (int d = 2; d >= 0; d--) m = (m << 1) | ((q[d] >> b) & 1u);
            key[k] = m;
      }
      perm.resize(n);
      for (int k = 0; k < n; k++) perm[k] = k;
      std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return key[a] < key[b]; });
}

// The MIXED mode runs on the bodies in Morton order of their initial
// positions: the inputs are permuted here, the outputs restored to the
// caller's order.
int lf_run(const struct ncgpu_leapfrog_args *a, int mode)
{
      Ctx &c = ctx();
      if (c.P.par_gravity_mode != NCGPU_GRAVITY_MIXED) return lf_core(a, mode, false);
      const int n = a->n;
      if (n <= 0 || !a->x0 || !a->v0 || !a->m || !a->R || !a->cm || a->nsteps < 0) return NCGPU_E_ARG;
      std::vector<int> perm;
      morton_order(a->x0, n, perm);
      const size_t N = (size_t)n;
      auto gather3 = [&](const double *src, std::vector<double> &dst) {
            dst.resize(3 * N);
            for (size_t i = 0; i < N; i++)
                  for (int d = 0; d < 3; d++) dst[3 * i + d] = src[3 * (size_t)perm[i] + d];
      };
      auto gather1 = [&](const double *src, std::vector<double> &dst) {
            dst.resize(N);
            for (size_t i = 0; i < N; i++) dst[i] = src[perm[i]];
      };
      std::vector<double> x0, v0, m, R, adj, tx0, tv0, tm, xf, vf, gx, gv, gm, txf;
      gather3(a->x0, x0); gather3(a->v0, v0); gather1(a->m, m); gather1(a->R, R);
      struct ncgpu_leapfrog_args b = *a;
      b.x0 = x0.data(); b.v0 = v0.data(); b.m = m.data(); b.R = R.data();
      if (a->adj_x_final) { gather3(a->adj_x_final, adj); b.adj_x_final = adj.data(); }
      if (a->tan_x0) { gather3(a->tan_x0, tx0); b.tan_x0 = tx0.data(); }
      if (a->tan_v0) { gather3(a->tan_v0, tv0); b.tan_v0 = tv0.data(); }
      if (a->tan_m) { gather1(a->tan_m, tm); b.tan_m = tm.data(); }
      if (a->x_final) { xf.resize(3 * N); b.x_final = xf.data(); }
      if (a->v_final) { vf.resize(3 * N); b.v_final = vf.data(); }
      if (a->grad_x0) { gx.resize(3 * N); b.grad_x0 = gx.data(); }
      if (a->grad_v0) { gv.resize(3 * N); b.grad_v0 = gv.data(); }
      if (a->grad_m) { gm.resize(N); b.grad_m = gm.data(); }
      if (a->tan_x_final) { txf.resize(3 * N); b.tan_x_final = txf.data(); }
      const int st = lf_core(&b, mode, true);
      if (st != NCGPU_OK) return st;
      auto scatter3 = [&](const std::vector<double> &src, double *dst) {
            for (size_t i = 0; i < N; i++)
                  for (int d = 0; d < 3; d++) dst[3 * (size_t)perm[i] + d] = src[3 * i + d];
      };
      if (a->x_final) scatter3(xf, a->x_final);
      if (a->v_final) scatter3(vf, a->v_final);
      if (a->grad_x0) scatter3(gx, a->grad_x0);
      if (a->grad_v0) scatter3(gv, a->grad_v0);
      if (a->grad_m)
            for (size_t i = 0; i < N; i++) a->grad_m[perm[i]] = gm[i];
      if (a->tan_x_final) scatter3(txf, a->tan_x_final);
      return NCGPU_OK;
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
