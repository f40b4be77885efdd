// Discrete adjoint and tangent-linear model of the fused stream-collide step
// (no reference counterpart). For one cell with pulled deviations g,
// rho = 1 + sum g, u = j/rho, P_p = 3 c_p.u + 4.5 (c_p.u)^2 - 1.5 |u|^2,
// e_p = w_p rho (1 + P_p) - w_p and f_p = g_p - omega (g_p - e_p):
//
//   adjoint   mu_q = (1 - omega) lam_q + omega (A - B.u + B.c_q),
//             A = sum_p w_p lam_p (1 + P_p),
//             B_a = 3 sum_p w_p lam_p c_pa (1 + 3 c_p.u) - 3 u_a sum_p w_p lam_p,
//             and reverse streaming lam_t,q(x - c_q) = mu_q(x);
// the adjoint buffers hold mu (the adjoint before its reverse streaming) at
// the cell that formed it, and the next adjoint step gathers
// lam_q(x) = mu_q(x + c_q): the forward's pull with the opposite shift, so
// every store is the cell's own and the shifted accesses are loads, as in the
// forward kernel;
//   dL/domega = sum over steps and cells of -lam.(g - e);
//   tangent   df_p = (1 - omega) dg_p + omega de_p + (e_p - g_p) domega,
//             de_p = w_p [(1 + P_p) drho + rho (3 (c_p.du)(1 + 3 c_p.u) - 3 u.du)],
//             drho = sum dg, du = (dj - u drho)/rho.
// The initial state f0_q = w_q P_q(u0) (rho = 1, the equilibrium of
// bgk_init_velocity) gives dL/du0 = B(lam_0, u0). The adjoint step evaluates
// rho, u and e of the forward state with fused multiply-adds; the tangent
// model uses the forward's own arithmetic (equilibrium<V>), so the two agree
// to the rounding of these terms.
//
// Kernels run a fixed grid (DIAG_BLOCKS x DIAG_THREADS) striding over the
// cells, and accumulate their sums into one compensated pair per block, so
// repeated runs give identical bits.
#include "kernels.h"
#include "reduce.cuh"

namespace bgk {

namespace {

__device__ __forceinline__ int wrapa(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// Adds the block's compensated sum v into its running pair acc[2*blk].
__device__ __forceinline__ void acc_block(KS v, KS* sh, double* acc) {
  const KS r = block_reduce(v, sh);
  if (threadIdx.x == 0) {
    KS a{acc[2 * blockIdx.x], acc[2 * blockIdx.x + 1]};
    kcomb(a, r);
    acc[2 * blockIdx.x] = a.s;
    acc[2 * blockIdx.x + 1] = a.c;
  }
}

template <class R>
__device__ __forceinline__ R cdot(int q, R ux, R uy, R uz) {
  return (R)cxq(q) * ux + (R)cyq(q) * uy + (R)czq(q) * uz;
}

template <class R>
__device__ __forceinline__ R wq(int q) {
  return wclass(q) == 0 ? (R)(1.0 / 3.0) : (wclass(q) == 1 ? (R)(1.0 / 18.0) : (R)(1.0 / 36.0));
}

template <class F>
__global__ void __launch_bounds__(DIAG_THREADS) k_adj_terminal(Pops<const typename F::S> f, Geo g,
                                                               const double* __restrict__ ut, Pops<typename F::S> lam,
                                                               double* acc) {
  using S = typename F::S; using V = typename F::V; using N = Num<V>;
  __shared__ KS sh[DIAG_THREADS];
  KS loss = {0.0, 0.0};
  const long long n = (long long)g.nx * g.ny * g.nz;
  const double invn = 1.0 / (double)n;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long long)g.nx * g.ny));
    const long long o = i + (long long)g.sx * (j + (long long)g.ny * k);
    V x[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) x[q] = V{f.p[q][o]};
    V e[Q], vx, vy, vz;
    const V rho = equilibrium<V>(x, e, vx, vy, vz);  // moments in the forward's order
    const double u[3] = {(double)N::raw(vx), (double)N::raw(vy), (double)N::raw(vz)};
    const double d[3] = {u[0] - ut[c], u[1] - ut[n + c], u[2] - ut[2 * n + c]};
    kadd(loss, 0.5 * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]));
    const double r = invn / (double)N::raw(rho);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const double l = r * (d[0] * (cxq(q) - u[0]) + d[1] * (cyq(q) - u[1]) + d[2] * (czq(q) - u[2]));
      // in the adjoint buffers' convention: lam_q(y) sits at y + c_q
      const long long oq = wrapa(i + cxq(q), g.nx) +
                           (long long)g.sx * (wrapa(j + cyq(q), g.ny) + (long long)g.ny * wrapa(k + czq(q), g.nz));
      lam.p[q][oq] = (S)l;
    }
  }
  acc_block(loss, sh, acc);
}

// One cell per thread on the forward kernels' launch shape, in one pass over
// the populations: with wl_p = w_p lam_p, the sums A, B and the dL/domega term
// need only the moments L0 = sum wl, M1 = sum wl c, M2 = sum wl c c^T and
// S1 = sum lam g of the cell, because P_p depends on c_p only through c_p.u:
//   A = L0 (1 + a) + 3 u.M1 + 4.5 u.M2.u,    a = -1.5 |u|^2,
//   B = 3 (M1 + 3 M2 u - u L0),
//   sum lam.(e - g) = rho A - L0 - S1.
// So no population array stays live across the cell. The forward state is
// pulled from x - c_q and lam gathered from x + c_q (lam_q(x) = mu_q(x + c_q)
// of the previous adjoint step), both as row loads like the forward kernel's;
// lam is read again from cache for the output, mu_q(x), stored at the cell.
// rho, u, the moment sums and A, B, G are formed in the form's arithmetic
// (double for FP64, float for FP32: in double the FP32 step was bound by the
// FP64 pipe rather than by its half-size loads); each cell's dL/domega term is
// added to the block's sum in double. Each block adds its dL/domega
// contribution (warp shuffles, then the four warp sums in order) into its
// own compensated pair acc[2*block].
template <class F>
__global__ void __launch_bounds__(128, 4) k_adj_step(Pops<const typename F::S> ft, Pops<const typename F::S> lin,
                                                     Pops<typename F::S> lout, Geo g, typename F::R omega,
                                                     double* acc) {
  using S = typename F::S; using R = typename F::R;
  using D = R;  // arithmetic of the moment sums: the form's (double for FP64, float for FP32)
  __shared__ double wsum[4];
  double dw = 0.0;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i < g.nx && j < g.ny) {
    const int im = i == 0 ? g.nx - 1 : i - 1, ip = i == g.nx - 1 ? 0 : i + 1;
    const int jm = j == 0 ? g.ny - 1 : j - 1, jp = j == g.ny - 1 ? 0 : j + 1;
    const int km = k == 0 ? g.nz - 1 : k - 1, kp = k == g.nz - 1 ? 0 : k + 1;
    const int o = i + g.sx * (j + g.ny * k);
    // s = +1: x - c_q (pull of the state); s = -1: x + c_q (gather of lam)
    auto offq = [&](int q, int s) {
      const int cx = s * cxq(q), cy = s * cyq(q), cz = s * czq(q);
      const int ii = cx > 0 ? im : (cx < 0 ? ip : i);
      const int jj = cy > 0 ? jm : (cy < 0 ? jp : j);
      const int kk = cz > 0 ? km : (cz < 0 ? kp : k);
      return ii + g.sx * (jj + g.ny * kk);
    };
    R rho = (R)1, jx = 0, jy = 0, jz = 0;
    D L0 = 0, m1x = 0, m1y = 0, m1z = 0, mxx = 0, myy = 0, mzz = 0, mxy = 0, mxz = 0, myz = 0, S1 = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const R x = (R)__ldg(ft.p[q] + offq(q, 1));
      const D lam = (D)__ldg(lin.p[q] + offq(q, -1));
      rho += x;
      jx += (R)cxq(q) * x;
      jy += (R)cyq(q) * x;
      jz += (R)czq(q) * x;
      S1 += lam * (D)x;
      const D wl = wq<D>(q) * lam;
      L0 += wl;
      m1x += cxq(q) * wl;
      m1y += cyq(q) * wl;
      m1z += czq(q) * wl;
      mxx += (cxq(q) * cxq(q)) * wl;
      myy += (cyq(q) * cyq(q)) * wl;
      mzz += (czq(q) * czq(q)) * wl;
      mxy += (cxq(q) * cyq(q)) * wl;
      mxz += (cxq(q) * czq(q)) * wl;
      myz += (cyq(q) * czq(q)) * wl;
    }
    const R ri = (R)1 / rho;
    const D ux = (D)(jx * ri), uy = (D)(jy * ri), uz = (D)(jz * ri);
    const D a = (D)-1.5 * (ux * ux + uy * uy + uz * uz);
    const D nx = mxx * ux + mxy * uy + mxz * uz;  // M2 u
    const D ny = mxy * ux + myy * uy + myz * uz;
    const D nz = mxz * ux + myz * uy + mzz * uz;
    const D A = L0 * ((D)1 + a) + (D)3 * (ux * m1x + uy * m1y + uz * m1z) + (D)4.5 * (ux * nx + uy * ny + uz * nz);
    const D Bx = (D)3 * (m1x + (D)3 * nx - ux * L0);
    const D By = (D)3 * (m1y + (D)3 * ny - uy * L0);
    const D Bz = (D)3 * (m1z + (D)3 * nz - uz * L0);
    const D G = A - (Bx * ux + By * uy + Bz * uz);
    dw = (double)((D)rho * A - L0 - S1);
    const R om1 = (R)1 - omega;
    const R om = omega;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const R lam = (R)__ldg(lin.p[q] + offq(q, -1));
      const R gq = (R)(G + cdot<D>(q, Bx, By, Bz));
      const R mu = om1 * lam + om * gq;
      lout.p[q][o] = (S)mu;  // mu_q(x): cell x - c_q of the next adjoint step gathers it as its lam_q
    }
  }
  // fixed-order block sum into this block's running pair
  for (int sft = 16; sft > 0; sft >>= 1) dw += __shfl_down_sync(0xffffffffu, dw, sft);
  const int t = threadIdx.x + blockDim.x * threadIdx.y;
  if ((t & 31) == 0) wsum[t >> 5] = dw;
  __syncthreads();
  if (t == 0) {
    double s = 0.0;
    for (int w = 0; w < 4; ++w) s += wsum[w];
    const long long b = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
    KS a2{acc[2 * b], acc[2 * b + 1]};
    kadd(a2, s);
    acc[2 * b] = a2.s;
    acc[2 * b + 1] = a2.c;
  }
}

// The adjoint step on a forward state rebuilt from the one after it, so that
// the backward pass reads no stored or recomputed state between checkpoints.
// The BGK update post = g - omega (g - e) keeps rho and j, so the
// post-collision populations x of a cell give e = e(rho, u) and the
// pre-collision ones g = (x - omega e) / (1 - omega); and since the state
// after the step holds post at the cell (f_{t+1}(x) = post_t(x)),
// sum lam.(e - g) = sum lam.(e - x) / (1 - omega). x is read unshifted from a
// stored forward state (FIRST: the checkpoint, or the final state, that ends
// the segment) or gathered from x + c_q of the g that the previous launch
// rebuilt (f_{t+1}(x)_q = g_{t+1}(x + c_q)_q, as g_{t+1} is the pull of
// f_{t+1}); lam is gathered at the same offsets. Writes mu(x) as k_adj_step
// does and, when store_g is set, the rebuilt g(x) for the next launch. The
// rebuilt state is the forward's up to rounding, which grows by up to
// 1 / |1 - omega| per rebuilt step in the non-equilibrium part: the driver
// uses this only where |1 - omega|^-(K-1) is small over a segment of K steps.
// Moment sums in the form's arithmetic, with fused multiply-adds, like
// k_adj_step; the dL/domega term of each cell is added in double. Register
// caps: 3 blocks/SM for FP64 (158 registers), 8 for FP32 (64); measured
// against 4 and 5 (FP64) and 4 and 6 (FP32), and against loading all 19
// lam before the moment loop, all slower.
template <class F, bool FIRST>
__global__ void __launch_bounds__(128, F::id == 0 ? 3 : 8)
    k_adj_inv(Pops<const typename F::S> fp, Pops<const typename F::S> lin, Pops<typename F::S> lout,
              Pops<typename F::S> gout, int store_g, Geo g, typename F::R omega, typename F::R rinv, double* acc) {
  using S = typename F::S; using R = typename F::R;
  using D = R;
  __shared__ double wsum[4];
  double dw = 0.0;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i < g.nx && j < g.ny) {
    const int im = i == 0 ? g.nx - 1 : i - 1, ip = i == g.nx - 1 ? 0 : i + 1;
    const int jm = j == 0 ? g.ny - 1 : j - 1, jp = j == g.ny - 1 ? 0 : j + 1;
    const int km = k == 0 ? g.nz - 1 : k - 1, kp = k == g.nz - 1 ? 0 : k + 1;
    const int o = i + g.sx * (j + g.ny * k);
    auto offp = [&](int q) {  // x + c_q
      const int ii = cxq(q) > 0 ? ip : (cxq(q) < 0 ? im : i);
      const int jj = cyq(q) > 0 ? jp : (cyq(q) < 0 ? jm : j);
      const int kk = czq(q) > 0 ? kp : (czq(q) < 0 ? km : k);
      return ii + g.sx * (jj + g.ny * kk);
    };
    R x[Q];
    R rho = (R)1, jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      x[q] = (R)__ldg(fp.p[q] + (FIRST ? o : offp(q)));
      rho += x[q];
      jx += (R)cxq(q) * x[q];
      jy += (R)cyq(q) * x[q];
      jz += (R)czq(q) * x[q];
    }
    const R ri = (R)1 / rho;
    const R ux = jx * ri, uy = jy * ri, uz = jz * ri;
    const R a = (R)-1.5 * (ux * ux + uy * uy + uz * uz);
    D L0 = 0, m1x = 0, m1y = 0, m1z = 0, mxx = 0, myy = 0, mzz = 0, mxy = 0, mxz = 0, myz = 0, S2 = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const D lam = (D)__ldg(lin.p[q] + offp(q));
      const R cu = cdot<R>(q, ux, uy, uz);
      const R e = wq<R>(q) * (rho * ((R)1 + a + cu * ((R)3 + (R)4.5 * cu)) - (R)1);
      if (store_g) gout.p[q][o] = (S)((x[q] - omega * e) * rinv);
      S2 += lam * (D)(e - x[q]);
      const D wl = wq<D>(q) * lam;
      L0 += wl;
      m1x += cxq(q) * wl;
      m1y += cyq(q) * wl;
      m1z += czq(q) * wl;
      mxx += (cxq(q) * cxq(q)) * wl;
      myy += (cyq(q) * cyq(q)) * wl;
      mzz += (czq(q) * czq(q)) * wl;
      mxy += (cxq(q) * cyq(q)) * wl;
      mxz += (cxq(q) * czq(q)) * wl;
      myz += (cyq(q) * czq(q)) * wl;
    }
    const D nx = mxx * ux + mxy * uy + mxz * uz;  // M2 u
    const D ny = mxy * ux + myy * uy + myz * uz;
    const D nz = mxz * ux + myz * uy + mzz * uz;
    const D A = L0 * ((D)1 + a) + (D)3 * (ux * m1x + uy * m1y + uz * m1z) + (D)4.5 * (ux * nx + uy * ny + uz * nz);
    const D Bx = (D)3 * (m1x + (D)3 * nx - ux * L0);
    const D By = (D)3 * (m1y + (D)3 * ny - uy * L0);
    const D Bz = (D)3 * (m1z + (D)3 * nz - uz * L0);
    const D G = A - (Bx * ux + By * uy + Bz * uz);
    dw = (double)S2 * (double)rinv;
    const R om1 = (R)1 - omega;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const R lam = (R)__ldg(lin.p[q] + offp(q));
      const R mu = om1 * lam + omega * (R)(G + cdot<D>(q, Bx, By, Bz));
      lout.p[q][o] = (S)mu;
    }
  }
  for (int sft = 16; sft > 0; sft >>= 1) dw += __shfl_down_sync(0xffffffffu, dw, sft);
  const int t = threadIdx.x + blockDim.x * threadIdx.y;
  if ((t & 31) == 0) wsum[t >> 5] = dw;
  __syncthreads();
  if (t == 0) {
    double s = 0.0;
    for (int w = 0; w < 4; ++w) s += wsum[w];
    const long long b = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
    KS a2{acc[2 * b], acc[2 * b + 1]};
    kadd(a2, s);
    acc[2 * b] = a2.s;
    acc[2 * b + 1] = a2.c;
  }
}

template <class F>
__global__ void __launch_bounds__(DIAG_THREADS) k_adj_grad_u0(Pops<const typename F::S> lam, Geo g,
                                                              const double* __restrict__ u0, double* grad) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long long)g.nx * g.ny));
    const double ux = u0[c], uy = u0[n + c], uz = u0[2 * n + c];
    double L0 = 0, Lx = 0, Ly = 0, Lz = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const long long oq = wrapa(i + cxq(q), g.nx) +
                           (long long)g.sx * (wrapa(j + cyq(q), g.ny) + (long long)g.ny * wrapa(k + czq(q), g.nz));
      const double wl = wq<double>(q) * (double)lam.p[q][oq];  // lam_q(y) = mu_q(y + c_q)
      const double t = wl * (1.0 + 3.0 * cdot<double>(q, ux, uy, uz));
      L0 += wl;
      Lx += t * cxq(q);
      Ly += t * cyq(q);
      Lz += t * czq(q);
    }
    grad[c] = 3.0 * Lx - 3.0 * ux * L0;
    grad[n + c] = 3.0 * Ly - 3.0 * uy * L0;
    grad[2 * n + c] = 3.0 * Lz - 3.0 * uz * L0;
  }
}

template <class F>
__global__ void __launch_bounds__(DIAG_THREADS) k_tan_init(Pops<typename F::S> df, Geo g,
                                                           const double* __restrict__ u0,
                                                           const double* __restrict__ du0) {
  using S = typename F::S;
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long long)g.nx * g.ny));
    const long long o = i + (long long)g.sx * (j + (long long)g.ny * k);
    const double ux = u0[c], uy = u0[n + c], uz = u0[2 * n + c];
    const double dx = du0[c], dy = du0[n + c], dz = du0[2 * n + c];
    const double udu = ux * dx + uy * dy + uz * dz;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const double cu = cdot<double>(q, ux, uy, uz), cdu = cdot<double>(q, dx, dy, dz);
      df.p[q][o] = (S)(wq<double>(q) * (3.0 * cdu * (1.0 + 3.0 * cu) - 3.0 * udu));
    }
  }
}

template <class F>
__global__ void __launch_bounds__(DIAG_THREADS) k_tan_step(Pops<const typename F::S> f, Pops<const typename F::S> df,
                                                           Pops<typename F::S> f2, Pops<typename F::S> df2, Geo g,
                                                           typename F::R omega, typename F::R domega) {
  using S = typename F::S; using R = typename F::R; using V = typename F::V; using N = Num<V>;
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long long)g.nx * g.ny));
    const long long o = i + (long long)g.sx * (j + (long long)g.ny * k);
    V x[Q];
    R dx[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int ii = wrapa(i - cxq(q), g.nx), jj = wrapa(j - cyq(q), g.ny), kk = wrapa(k - czq(q), g.nz);
      const long long off = ii + (long long)g.sx * (jj + (long long)g.ny * kk);
      x[q] = V{f.p[q][off]};
      dx[q] = (R)df.p[q][off];
    }
    V e[Q], vx, vy, vz;
    const V rhov = equilibrium<V>(x, e, vx, vy, vz);
    const R rho = N::raw(rhov), ux = N::raw(vx), uy = N::raw(vy), uz = N::raw(vz);
    const R usq = ux * ux + uy * uy + uz * uz;
    R drho = 0, djx = 0, djy = 0, djz = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      drho += dx[q];
      djx += (R)cxq(q) * dx[q];
      djy += (R)cyq(q) * dx[q];
      djz += (R)czq(q) * dx[q];
    }
    const R dux = (djx - ux * drho) / rho, duy = (djy - uy * drho) / rho, duz = (djz - uz * drho) / rho;
    const R udu = ux * dux + uy * duy + uz * duz;
    const R om1 = (R)1 - omega;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const R cu = cdot<R>(q, ux, uy, uz), cdu = cdot<R>(q, dux, duy, duz);
      const R P = (R)3 * cu + (R)4.5 * cu * cu - (R)1.5 * usq;
      const R de = wq<R>(q) * (((R)1 + P) * drho + rho * ((R)3 * cdu * ((R)1 + (R)3 * cu) - (R)3 * udu));
      df2.p[q][o] = (S)(om1 * dx[q] + omega * de + (N::raw(e[q]) - N::raw(x[q])) * domega);
    }
    collide<V>(x, V{omega});
#pragma unroll
    for (int q = 0; q < Q; ++q) f2.p[q][o] = N::raw(x[q]);
  }
}

template <class F>
__global__ void __launch_bounds__(DIAG_THREADS) k_tan_loss(Pops<const typename F::S> f, Pops<const typename F::S> df,
                                                           Geo g, const double* __restrict__ ut, double* acc) {
  using V = typename F::V; using N = Num<V>;
  __shared__ KS sh[DIAG_THREADS];
  KS dl = {0.0, 0.0};
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long long)g.nx * g.ny));
    const long long o = i + (long long)g.sx * (j + (long long)g.ny * k);
    V x[Q];
    double drho = 0, djx = 0, djy = 0, djz = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      x[q] = V{f.p[q][o]};
      const double d = (double)df.p[q][o];
      drho += d;
      djx += cxq(q) * d;
      djy += cyq(q) * d;
      djz += czq(q) * d;
    }
    V e[Q], vx, vy, vz;
    const double rho = (double)N::raw(equilibrium<V>(x, e, vx, vy, vz));
    const double u[3] = {(double)N::raw(vx), (double)N::raw(vy), (double)N::raw(vz)};
    const double du[3] = {(djx - u[0] * drho) / rho, (djy - u[1] * drho) / rho, (djz - u[2] * drho) / rho};
    kadd(dl, (u[0] - ut[c]) * du[0] + (u[1] - ut[n + c]) * du[1] + (u[2] - ut[2 * n + c]) * du[2]);
  }
  acc_block(dl, sh, acc);
}

__global__ void __launch_bounds__(DIAG_THREADS) k_acc_total(const double* __restrict__ acc, double* total) {
  __shared__ KS sh[DIAG_THREADS];
  KS a = {0.0, 0.0};
  for (int b = threadIdx.x; b < DIAG_BLOCKS; b += blockDim.x) kcomb(a, KS{acc[2 * b], acc[2 * b + 1]});
  const KS r = block_reduce(a, sh);
  if (threadIdx.x == 0) *total = __dadd_rn(r.s, r.c);
}

// Launch shape of the adjoint step (x rows in blockDim.x, 128 threads).
void adj_shape(const Geo& g, dim3* grid, dim3* block) {
  const int tx = g.nx >= 128 ? 128 : ((g.nx + 31) / 32) * 32;
  const int ty = 128 / tx;
  *block = dim3(tx, ty, 1);
  *grid = dim3((g.nx + tx - 1) / tx, (g.ny + ty - 1) / ty, g.nz);
}

// Sums n compensated pairs in a fixed order into *total.
__global__ void __launch_bounds__(DIAG_THREADS) k_acc_total_n(const double* __restrict__ acc, long long n,
                                                              double* total) {
  __shared__ KS sh[DIAG_THREADS];
  KS a = {0.0, 0.0};
  for (long long b = threadIdx.x; b < n; b += blockDim.x) kcomb(a, KS{acc[2 * b], acc[2 * b + 1]});
  const KS r = block_reduce(a, sh);
  if (threadIdx.x == 0) *total = __dadd_rn(r.s, r.c);
}

template <class S> Pops<S> pops(const Lattice& L) {
  Pops<S> p;
  for (int q = 0; q < Q; ++q) p.p[q] = (S*)L.p[q];
  return p;
}

}  // namespace

#define BGK_FORM_DISPATCH(L, CALL64, CALL32)      \
  switch ((L).form) {                             \
    case FORM_F64: CALL64; return cudaGetLastError(); \
    case FORM_F32: CALL32; return cudaGetLastError(); \
  }                                               \
  return cudaErrorInvalidValue;

cudaError_t launch_adj_terminal(const Lattice& f, const double* ut, const Lattice& lam, double* acc, cudaStream_t st) {
  BGK_FORM_DISPATCH(f,
      (k_adj_terminal<F64><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(pops<const double>(f), f.g, ut, pops<double>(lam), acc)),
      (k_adj_terminal<F32><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(pops<const float>(f), f.g, ut, pops<float>(lam), acc)))
}

long long adj_step_blocks(const Geo& g) {
  dim3 grid, block;
  adj_shape(g, &grid, &block);
  return (long long)grid.x * grid.y * grid.z;
}

cudaError_t launch_adj_step(const Lattice& ft, const Lattice& lin, const Lattice& lout, double omega, double* acc,
                            cudaStream_t st) {
  dim3 grid, block;
  adj_shape(ft.g, &grid, &block);
  BGK_FORM_DISPATCH(ft,
      (k_adj_step<F64><<<grid, block, 0, st>>>(pops<const double>(ft), pops<const double>(lin), pops<double>(lout),
                                               ft.g, omega, acc)),
      (k_adj_step<F32><<<grid, block, 0, st>>>(pops<const float>(ft), pops<const float>(lin), pops<float>(lout),
                                               ft.g, (float)omega, acc)))
}

cudaError_t launch_adj_inv(const Lattice& post, bool first, const Lattice& lin, const Lattice& lout,
                           const Lattice* gout, double omega, double* acc, cudaStream_t st) {
  dim3 grid, block;
  adj_shape(post.g, &grid, &block);
  const int sg = gout != nullptr;
  const Lattice& go = gout ? *gout : lout;  // not written when sg = 0
  const double rinv = 1.0 / (1.0 - omega);
  switch (post.form) {
    case FORM_F64: {
      auto kf = first ? k_adj_inv<F64, true> : k_adj_inv<F64, false>;
      kf<<<grid, block, 0, st>>>(pops<const double>(post), pops<const double>(lin), pops<double>(lout),
                                 pops<double>(go), sg, post.g, omega, rinv, acc);
      return cudaGetLastError();
    }
    case FORM_F32: {
      auto kf = first ? k_adj_inv<F32, true> : k_adj_inv<F32, false>;
      kf<<<grid, block, 0, st>>>(pops<const float>(post), pops<const float>(lin), pops<float>(lout),
                                 pops<float>(go), sg, post.g, (float)omega, (float)rinv, acc);
      return cudaGetLastError();
    }
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_acc_total_n(const double* acc, long long n, double* total, cudaStream_t st) {
  k_acc_total_n<<<1, DIAG_THREADS, 0, st>>>(acc, n, total);
  return cudaGetLastError();
}

cudaError_t launch_adj_grad_u0(const Lattice& lam0, const double* u0, double* grad, cudaStream_t st) {
  BGK_FORM_DISPATCH(lam0,
      (k_adj_grad_u0<F64><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(pops<const double>(lam0), lam0.g, u0, grad)),
      (k_adj_grad_u0<F32><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(pops<const float>(lam0), lam0.g, u0, grad)))
}

cudaError_t launch_tan_init(const Lattice& df, const double* u0, const double* du0, cudaStream_t st) {
  BGK_FORM_DISPATCH(df,
      (k_tan_init<F64><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(pops<double>(df), df.g, u0, du0)),
      (k_tan_init<F32><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(pops<float>(df), df.g, u0, du0)))
}

cudaError_t launch_tan_step(const Lattice& f, const Lattice& df, const Lattice& f2, const Lattice& df2, double omega,
                            double domega, cudaStream_t st) {
  BGK_FORM_DISPATCH(f,
      (k_tan_step<F64><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(pops<const double>(f), pops<const double>(df),
                                                             pops<double>(f2), pops<double>(df2), f.g, omega,
                                                             domega)),
      (k_tan_step<F32><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(pops<const float>(f), pops<const float>(df),
                                                             pops<float>(f2), pops<float>(df2), f.g, (float)omega,
                                                             (float)domega)))
}

cudaError_t launch_tan_loss(const Lattice& f, const Lattice& df, const double* ut, double* acc, cudaStream_t st) {
  BGK_FORM_DISPATCH(f,
      (k_tan_loss<F64><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(pops<const double>(f), pops<const double>(df), f.g, ut,
                                                             acc)),
      (k_tan_loss<F32><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(pops<const float>(f), pops<const float>(df), f.g, ut,
                                                             acc)))
}

cudaError_t launch_acc_total(const double* acc, double* total, cudaStream_t st) {
  k_acc_total<<<1, DIAG_THREADS, 0, st>>>(acc, total);
  return cudaGetLastError();
}

}  // namespace bgk
