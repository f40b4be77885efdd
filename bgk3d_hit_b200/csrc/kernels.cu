// CUDA kernels of the BGK3D_HIT hot path for sm_100a.
//
//   k_two        fused pull-stream + BGK collide, two lattices, pop 19 in place
//                (SRC/col_MC.F90:98-421); periodic wrap by index arithmetic
//                replaces the halo exchange of SRC/bcond.comm.step3.F90
//   k_aa         in-place AA-pattern variant of the same update (no reference
//                counterpart; same per-cell arithmetic)
//   k_two_f32v, k_aa_f32v / k_two_f16v, k_aa_f16v
//                the same updates with two FP32 / four FP16 cells of a row per
//                thread (8-byte accesses, x-crossing values by warp shuffle);
//                the defaults of those forms where a box fits them
//   k_aa_f16w, k_aa_f32w
//                the AA odd step with eight FP16 (BGK) / four FP32 (BGK and
//                Smagorinsky) cells per thread, 16-byte accesses: its default
//                where a box fits it
//   k_slab       two-lattice step of one z-slab with the face exchange fused in
//   k_init_*     equilibrium initial conditions (SRC/init.F90:83-141)
//   k_diag       diagno + dissipation + strain-rate sums (SRC/diagno.F90:73-121,
//                SRC/dissipation.F90:65-269) as deterministic compensated
//                per-block partials
//   k_enstrophy  0.5|curl u|^2 from the local velocity field
//   k_shift3     shift-only stencil of SRC/do_somethingGPU.F90:37-100
#include "kernels.h"
#include "reduce.cuh"

namespace bgk {

__device__ __forceinline__ int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

__device__ __forceinline__ double ldg(const double* p) { return __ldg(p); }
__device__ __forceinline__ float ldg(const float* p) { return __ldg(p); }
__device__ __forceinline__ __half ldg(const __half* p) { return __ldg(p); }

// Moments of 19 local deviations in the reference's order
// (SRC/diagno.F90:96-104, identical to SRC/col_MC.F90:133-141).
template <class V>
__device__ __forceinline__ V moments(const V (&x)[Q], V& vx, V& vy, V& vz) {
  using N = Num<V>;
  const V uno = N::c(1.0), cte1 = N::c(1.0);
  V rho = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7]
        + x[8] + x[9] + x[10] + x[11] + x[12] + x[13] + x[14] + x[15]
        + x[16] + x[17] + x[18] + cte1;
  V rhoinv = uno / rho;
  vx = (x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]) * rhoinv;
  vy = (x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]) * rhoinv;
  vz = (x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]) * rhoinv;
  return rho;
}

// Launch shape of the per-cell stream kernels: x-rows in blockDim.x.
struct Shape { dim3 grid, block; };
static Shape cell_shape(const Geo& g) {
  int tx = g.nx >= 128 ? 128 : ((g.nx + 31) / 32) * 32;
  int ty = 256 / tx;
  Shape s;
  s.block = dim3(tx, ty, 1);
  s.grid = dim3((g.nx + tx - 1) / tx, (g.ny + ty - 1) / ty, g.nz);
  return s;
}

static int grid_1d(long long n, int threads, int cap) {
  long long b = (n + threads - 1) / threads;
  return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

// ------------------------------------------------------------- two lattice
template <class F, bool LES = false>
__global__ void __launch_bounds__(256) k_two(Pops<const typename F::S> src, Pops<typename F::S> dst, Geo g, StepK K) {
  using S = typename F::S;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const int im = i == 0 ? g.nx - 1 : i - 1, ip = i == g.nx - 1 ? 0 : i + 1;
  const int jm = j == 0 ? g.ny - 1 : j - 1, jp = j == g.ny - 1 ? 0 : j + 1;
  const int km = k == 0 ? g.nz - 1 : k - 1, kp = k == g.nz - 1 ? 0 : k + 1;
  S v[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    // pull from (i - cx, j - cy, k - cz), SRC/col_MC.F90:113-131
    const int ii = cxq(q) > 0 ? im : (cxq(q) < 0 ? ip : i);
    const int jj = cyq(q) > 0 ? jm : (cyq(q) < 0 ? jp : j);
    const int kk = czq(q) > 0 ? km : (czq(q) < 0 ? kp : k);
    const int off = ii + g.sx * (jj + g.ny * kk);
    // pop 19 with a plain load: in the time loop it is updated in place
    // (src.p[18] == dst.p[18]); the adjoint's out-of-place steps pass distinct arrays
    v[q] = (q == Q - 1) ? src.p[Q - 1][off] : ldg(src.p[q] + off);
  }
  F::template cell<LES>(v, K);
  const int o = i + g.sx * (j + g.ny * k);
#pragma unroll
  for (int q = 0; q < Q; ++q) dst.p[q][o] = v[q];
}

// FP16 two-lattice step with 4 cells per thread and 8-byte accesses. A row of
// nx cells is handled by tpr = nx/4 consecutive threads (tpr a power of two).
// x-shifted pulls take the element that crosses a thread boundary from the
// neighbouring lane (warp shuffle); across warp boundaries (tpr > 32) lanes 0
// and 31 load it. Each cell's arithmetic is F16::cell's (moments16, pair16,
// rest16). The collision runs on two cells at a time, their outputs replacing
// their inputs in the packed registers, and the kernel runs 128-thread blocks
// at 96 registers (5 blocks per SM, no spills). On B200 at 256^3, with every
// row load issued before the shuffles, that measured 84.4 GLUPS against 82.0
// capped at 80 registers (6 blocks per SM, 52 spilled bytes; the Smagorinsky
// variant 78.5 against 67.9 with 108 spilled bytes); earlier forms of the
// kernel measured 76.6 with 256-thread blocks, 64.5 for all four cells at once
// at 2 blocks per SM and 58.4 at 64 registers (heavy spills).
__device__ __forceinline__ unsigned short ldg_u16(const __half* p) {
  return __ldg(reinterpret_cast<const unsigned short*>(p));
}
__device__ __forceinline__ unsigned h2u(__half2 h) { return *reinterpret_cast<unsigned*>(&h); }
__device__ __forceinline__ float2 u2f2(unsigned u) { return __half22float2(*reinterpret_cast<__half2*>(&u)); }

// Collision of four FP16 cells packed in Y (population q of cell m in half m
// of Y[q]), F16::cell's arithmetic, on cells 0, 1 (low words) then cells 2, 3
// (high words): each half's outputs replace its inputs in Y, so only two
// cells' moments are live at a time. LES: the Smagorinsky collision
// (moments16_les: per-cell relaxation constants, the same pair update).
template <bool LES>
__device__ __forceinline__ void collide4_f16(uint2 (&Y)[Q], const StepK& K) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    Mom16 M[2];
    float om1[2] = {K.om1, K.om1};
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      float y[Q];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const float2 f = u2f2(h ? Y[q].y : Y[q].x);
        y[q] = m ? f.y : f.x;
      }
      if constexpr (LES) M[m] = moments16_les(y, K, om1[m]);
      else M[m] = moments16(y, K);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const int r = oppq(q);
      const float2 a = u2f2(h ? Y[q].y : Y[q].x), c = u2f2(h ? Y[r].y : Y[r].x);
      float p0, p1, o0, o1;
      pair16(q, a.x, c.x, M[0], om1[0], p0, o0);
      pair16(q, a.y, c.y, M[1], om1[1], p1, o1);
      const unsigned pq = h2u(__floats2half2_rn(p0, p1)), pr = h2u(__floats2half2_rn(o0, o1));
      if (h) { Y[q].y = pq; Y[r].y = pr; } else { Y[q].x = pq; Y[r].x = pr; }
    }
    {
      const float2 a = u2f2(h ? Y[Q - 1].y : Y[Q - 1].x);
      const unsigned pz = h2u(__floats2half2_rn(rest16(a.x, M[0], om1[0]), rest16(a.y, M[1], om1[1])));
      if (h) Y[Q - 1].y = pz; else Y[Q - 1].x = pz;
    }
  }
}

// Lanes that exchange x-neighbours in the several-cells-per-thread kernels:
// a row of nx cells is tpr = nx/V consecutive threads (V cells per thread).
// Rows shorter than a warp wrap inside it; rows of one or more warps wrap
// through global memory at the warp's first / last lane (edge_prev /
// edge_next).
struct XLanes {
  int src_prev, src_next;
  bool edge_prev, edge_next;
  __device__ XLanes(int tpr, int pos, int lane) {
    edge_prev = edge_next = false;
    if (tpr >= 32) {
      src_prev = (lane + 31) & 31;
      src_next = (lane + 1) & 31;
      edge_prev = lane == 0;
      edge_next = lane == 31;
    } else {
      src_prev = pos == 0 ? lane + tpr - 1 : lane - 1;
      src_next = pos == tpr - 1 ? lane - tpr + 1 : lane + 1;
    }
  }
};

// Second half of the x-shifted row loads of the four-cells-per-thread FP16
// kernels. Y[q] holds the aligned chunk of elements i0..i0+3 of population
// q's source row; cells i0..i0+3 need elements i0 - cx ... i0 + 3 - cx with
// cx = c_q,x, so the element that crosses the chunk boundary comes from the
// neighbouring lane (warp shuffle) or, for a warp's edge lane, from E[q],
// which that lane loaded together with the chunks. All loads are issued
// before the first shuffle: measured on B200 (FP16 AA odd step, 256^3), this
// ordering lifted the pair of AA steps from 72.2 to 75.6 GLUPS.
__device__ __forceinline__ void shift_rows(uint2 (&Y)[Q], const unsigned short (&E)[Q], const XLanes& xl) {
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const uint2 A = Y[q];
    if (cxq(q) > 0) {  // elements i0-1 .. i0+2
      unsigned prev = __shfl_sync(0xffffffffu, A.y >> 16, xl.src_prev);
      if (xl.edge_prev) prev = E[q];
      Y[q].x = __byte_perm(A.x, prev, 0x1054);
      Y[q].y = __byte_perm(A.x, A.y, 0x5432);
    } else if (cxq(q) < 0) {  // elements i0+1 .. i0+4
      unsigned next = __shfl_sync(0xffffffffu, A.x & 0xffffu, xl.src_next);
      if (xl.edge_next) next = E[q];
      Y[q].x = __byte_perm(A.x, A.y, 0x5432);
      Y[q].y = __byte_perm(A.y, next, 0x5432);
    }
  }
}

template <bool LES>
__global__ void __launch_bounds__(128, 5) k_two_f16v(Pops<const __half> src, Pops<__half> dst, Geo g, StepK K,
                                                  int log_tpr, int k0) {
  const int tpr = 1 << log_tpr;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = t >> log_tpr, pos = t & (tpr - 1);
  const int k = blockIdx.y + k0;  // planes k0 .. k0 + gridDim.y - 1
  if (j >= g.ny) return;  // whole warps: ny*tpr is a multiple of 32
  const XLanes xl(tpr, pos, threadIdx.x & 31);
  const int i0 = pos * 4;
  const int jm = j == 0 ? g.ny - 1 : j - 1, jp = j == g.ny - 1 ? 0 : j + 1;
  const int km = k == 0 ? g.nz - 1 : k - 1, kp = k == g.nz - 1 ? 0 : k + 1;
  const int i_prev = pos == 0 ? g.nx - 1 : i0 - 1;
  const int i_next = pos == tpr - 1 ? 0 : i0 + 4;
  uint2 Y[Q];  // four cells' stored values per population, cell m in half m
  unsigned short E[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int jj = cyq(q) > 0 ? jm : (cyq(q) < 0 ? jp : j);
    const int kk = czq(q) > 0 ? km : (czq(q) < 0 ? kp : k);
    const __half* p = (q == Q - 1 ? (const __half*)dst.p[Q - 1] : src.p[q]) + g.sx * (jj + g.ny * kk);
    Y[q] = (q == Q - 1) ? *reinterpret_cast<const uint2*>(p + i0) : __ldg(reinterpret_cast<const uint2*>(p + i0));
    E[q] = 0;
    if (cxq(q) > 0 && xl.edge_prev) E[q] = ldg_u16(p + i_prev);
    if (cxq(q) < 0 && xl.edge_next) E[q] = ldg_u16(p + i_next);
  }
  shift_rows(Y, E, xl);
  collide4_f16<LES>(Y, K);
  const int o = i0 + g.sx * (j + g.ny * k);
#pragma unroll
  for (int q = 0; q < Q; ++q) *reinterpret_cast<uint2*>(dst.p[q] + o) = Y[q];
}

// Second half of the x-shifted row loads of the two-cells-per-thread FP32
// kernels: shift_rows on chunks of two floats (Y[q] holds elements i0, i0+1;
// the element that crosses the chunk comes from the neighbouring lane or, for
// a warp's edge lane, from E[q]).
__device__ __forceinline__ void shift_rows_f32(float2 (&Y)[Q], const float (&E)[Q], const XLanes& xl) {
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const float2 A = Y[q];
    if (cxq(q) > 0) {  // elements i0-1, i0
      float prev = __shfl_sync(0xffffffffu, A.y, xl.src_prev);
      if (xl.edge_prev) prev = E[q];
      Y[q] = make_float2(prev, A.x);
    } else if (cxq(q) < 0) {  // elements i0+1, i0+2
      float next = __shfl_sync(0xffffffffu, A.x, xl.src_next);
      if (xl.edge_next) next = E[q];
      Y[q] = make_float2(A.y, next);
    }
  }
}

// FP32 two-lattice step with 2 cells per thread and 8-byte accesses (tpr =
// nx/2 threads per row): k_two_f16v's row split and x-crossing shuffles on
// chunks of two floats, F32::cell's arithmetic on each cell, so the results
// are those of k_two<F32>. 72 registers (80 for the Smagorinsky step), no
// spills.
template <bool LES>
__global__ void __launch_bounds__(128, 5) k_two_f32v(Pops<const float> src, Pops<float> dst, Geo g, StepK K,
                                                  int log_tpr, int k0) {
  const int tpr = 1 << log_tpr;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = t >> log_tpr, pos = t & (tpr - 1);
  const int k = blockIdx.y + k0;  // planes k0 .. k0 + gridDim.y - 1
  if (j >= g.ny) return;  // whole warps: ny*tpr is a multiple of 32
  const XLanes xl(tpr, pos, threadIdx.x & 31);
  const int i0 = pos * 2;
  const int jm = j == 0 ? g.ny - 1 : j - 1, jp = j == g.ny - 1 ? 0 : j + 1;
  const int km = k == 0 ? g.nz - 1 : k - 1, kp = k == g.nz - 1 ? 0 : k + 1;
  const int i_prev = pos == 0 ? g.nx - 1 : i0 - 1;
  const int i_next = pos == tpr - 1 ? 0 : i0 + 2;
  float2 Y[Q];  // two cells' values per population, cell m in component m
  float E[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int jj = cyq(q) > 0 ? jm : (cyq(q) < 0 ? jp : j);
    const int kk = czq(q) > 0 ? km : (czq(q) < 0 ? kp : k);
    // pop 19 with a plain load: in the time loop it is updated in place
    // (src.p[18] == dst.p[18]); the adjoint's out-of-place steps pass distinct arrays
    const float* p = src.p[q] + g.sx * (jj + g.ny * kk);
    Y[q] = (q == Q - 1) ? *reinterpret_cast<const float2*>(p + i0) : __ldg(reinterpret_cast<const float2*>(p + i0));
    E[q] = 0.f;
    if (cxq(q) > 0 && xl.edge_prev) E[q] = __ldg(p + i_prev);
    if (cxq(q) < 0 && xl.edge_next) E[q] = __ldg(p + i_next);
  }
  shift_rows_f32(Y, E, xl);
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    float s[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) s[q] = m ? Y[q].y : Y[q].x;
    F32::cell<LES>(s, K);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if (m) Y[q].y = s[q];
      else Y[q].x = s[q];
    }
  }
  const int o = i0 + g.sx * (j + g.ny * k);
#pragma unroll
  for (int q = 0; q < Q; ++q) *reinterpret_cast<float2*>(dst.p[q] + o) = Y[q];
}

// FP16 two-lattice step with 2 cells per thread and 4-byte accesses (tpr =
// nx/2 threads per row); otherwise as k_two_f16v.
__global__ void __launch_bounds__(256, 4) k_two_f16v2(Pops<const __half> src, Pops<__half> dst, Geo g, StepK K,
                                                   int log_tpr) {
  const int tpr = 1 << log_tpr;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = t >> log_tpr, pos = t & (tpr - 1);
  const int k = blockIdx.y;
  if (j >= g.ny) return;  // whole warps: ny*tpr is a multiple of 32
  const int lane = threadIdx.x & 31;
  const int i0 = pos * 2;
  const int jm = j == 0 ? g.ny - 1 : j - 1, jp = j == g.ny - 1 ? 0 : j + 1;
  const int km = k == 0 ? g.nz - 1 : k - 1, kp = k == g.nz - 1 ? 0 : k + 1;
  int src_prev, src_next;
  bool load_prev = false, load_next = false;
  if (tpr >= 32) {
    src_prev = (lane + 31) & 31;
    src_next = (lane + 1) & 31;
    load_prev = lane == 0;
    load_next = lane == 31;
  } else {
    src_prev = pos == 0 ? lane + tpr - 1 : lane - 1;
    src_next = pos == tpr - 1 ? lane - tpr + 1 : lane + 1;
  }
  const int i_prev = pos == 0 ? g.nx - 1 : i0 - 1;
  const int i_next = pos == tpr - 1 ? 0 : i0 + 2;
  unsigned Y[Q];  // two cells' stored values per population, cell m in half m
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int jj = cyq(q) > 0 ? jm : (cyq(q) < 0 ? jp : j);
    const int kk = czq(q) > 0 ? km : (czq(q) < 0 ? kp : k);
    const __half* p = (q == Q - 1 ? (const __half*)dst.p[Q - 1] : src.p[q]) + g.sx * (jj + g.ny * kk);
    const unsigned A = (q == Q - 1) ? *reinterpret_cast<const unsigned*>(p + i0)
                                    : __ldg(reinterpret_cast<const unsigned*>(p + i0));
    if (cxq(q) == 0) {
      Y[q] = A;
    } else if (cxq(q) > 0) {  // cells need elements i0-1, i0
      unsigned prev = __shfl_sync(0xffffffffu, A >> 16, src_prev);
      if (load_prev) prev = ldg_u16(p + i_prev);
      Y[q] = __byte_perm(A, prev, 0x1054);
    } else {  // cells need elements i0+1, i0+2
      unsigned next = __shfl_sync(0xffffffffu, A & 0xffffu, src_next);
      if (load_next) next = ldg_u16(p + i_next);
      Y[q] = __byte_perm(A, next, 0x5432);
    }
  }
  Mom16 M[2];
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    float y[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const float2 f = u2f2(Y[q]);
      y[q] = m ? f.y : f.x;
    }
    M[m] = moments16(y, K);
  }
  const int o = i0 + g.sx * (j + g.ny * k);
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    const int r = oppq(q);
    const float2 a = u2f2(Y[q]), c = u2f2(Y[r]);
    float p0, p1, o0, o1;
    pair16(q, a.x, c.x, M[0], K.om1, p0, o0);
    pair16(q, a.y, c.y, M[1], K.om1, p1, o1);
    *reinterpret_cast<unsigned*>(dst.p[q] + o) = h2u(__floats2half2_rn(p0, p1));
    *reinterpret_cast<unsigned*>(dst.p[r] + o) = h2u(__floats2half2_rn(o0, o1));
  }
  {
    const float2 a = u2f2(Y[Q - 1]);
    *reinterpret_cast<unsigned*>(dst.p[Q - 1] + o) =
        h2u(__floats2half2_rn(rest16(a.x, M[0], K.om1), rest16(a.y, M[1], K.om1)));
  }
}

// --------------------------------------------------------------- AA pattern
// Even step: g_q(x) = slot q at x; result q -> slot opp(q) at x.
// Odd step:  g_q(x) = slot opp(q) at x - c_q; result q -> slot q at x + c_q.
// Each thread reads exactly the locations it writes, so the update is
// race-free in place; a location is never read after it has been written,
// which also makes the read-only load path safe.
template <class F, bool ODD, bool LES>
__device__ __forceinline__ void aa_cell(Pops<typename F::S>& a, const Geo& g, const StepK& K) {
  using S = typename F::S;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const int o = i + g.sx * (j + g.ny * k);
  const int im = i == 0 ? g.nx - 1 : i - 1, ip = i == g.nx - 1 ? 0 : i + 1;
  const int jm = j == 0 ? g.ny - 1 : j - 1, jp = j == g.ny - 1 ? 0 : j + 1;
  const int km = k == 0 ? g.nz - 1 : k - 1, kp = k == g.nz - 1 ? 0 : k + 1;
  // location x - c_q (read, slot opp(q)) == location x + c_opp(q) (write, slot opp(q))
  auto back = [&](int q) {
    const int ii = cxq(q) > 0 ? im : (cxq(q) < 0 ? ip : i);
    const int jj = cyq(q) > 0 ? jm : (cyq(q) < 0 ? jp : j);
    const int kk = czq(q) > 0 ? km : (czq(q) < 0 ? kp : k);
    return ii + g.sx * (jj + g.ny * kk);
  };
  S v[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) v[q] = ODD ? ldg(a.p[oppq(q)] + back(q)) : ldg(a.p[q] + o);
  F::template cell<LES>(v, K);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    if (ODD) a.p[q][back(oppq(q))] = v[q];
    else a.p[oppq(q)][o] = v[q];
  }
}

template <class F, bool ODD, bool LES = false>
__global__ void __launch_bounds__(256) k_aa(Pops<typename F::S> a, Geo g, StepK K) {
  aa_cell<F, ODD, LES>(a, g, K);
}

// The FP16 odd step (BGK) is latency-bound on registers: capped at 48 (5
// blocks per SM) it measured 53.7 against 50.4 GLUPS uncapped for that step at
// 256^3 on B200, a few spilled bytes included.
__global__ void __launch_bounds__(256, 5) k_aa_f16_odd(Pops<__half> a, Geo g, StepK K) {
  aa_cell<F16, true, false>(a, g, K);
}

// FP16 AA pattern with four cells per thread (the same row split, shuffles
// and collision as k_two_f16v). Even step: slot q at x -> slot opp(q) at x,
// 8-byte accesses, no exchange. Odd step: slot opp(q) at x - c_q -> slot q at
// x + c_q, with the x-crossing values moved between lanes on both the load and
// the store side; on the store side a warp-edge lane gets its crossing value
// from the neighbouring warp of the block through shared memory after a block
// barrier, so only block boundaries need partial stores (a warp edge with 2-
// and 4-byte stores costs about as much as the rest of the warp's stores of
// that population: 240 -> 223 us per 256^3 odd step, AA pair 77.1 -> 80.1
// GLUPS). Every (location, slot) pair is still read and written by the
// thread of the cell that owns it in the one-cell-per-thread kernel, or by a
// lane of the same warp after a shuffle that orders it behind the owner's
// loads, or by a lane of another warp of the block after the barrier that
// follows every warp's loads, so the in-place update stays race-free.
// 128-thread blocks at 96 registers (5 blocks per SM) like k_two_f16v. The odd step stores to the
// rows it loaded from; left alone, the compiler keeps those 18 row addresses
// live through the collision, so the BGK odd step recomputes them from an
// opaque copy of (j, k) and fits 96 registers without spills (5 blocks per
// SM). On B200 at 256^3 the pair of steps measured 72.3 GLUPS, against 71.1
// with the addresses kept (128 registers, 4 blocks), 69.5 with 256-thread
// blocks, 63.4 with the odd step capped at 80 registers (282 spilled bytes),
// 62.8-65.0 with two cells per thread on the odd step, and 58 for one cell per
// thread; with the loads issued before the shuffles and the even step at 96
// registers as well, 76.9. The LES odd step recomputes its store rows the
// same way (96 registers, a few spilled bytes).
// Store side of the AA odd step: stores four cells' values Y (cells
// i0..i0+3) at elements i0 + cx ... i0 + 3 + cx of row p as one aligned
// 8-byte chunk, completed with the neighbouring lane's crossing value (warp
// shuffle). A warp-edge lane takes that value from the neighbouring warp
// through shared memory (from_prev / from_next) when that warp is in the same
// block (prev_in / next_in) and stores its whole chunk, the neighbour then
// skipping its store of the crossing element; at block boundaries the edge
// lanes store their part of the chunk and their crossing value with 4- and
// 2-byte stores.
__device__ __forceinline__ void shift_out(uint2 Y, int cx, __half* p, int i0, int i_prev, int i_next,
                                              const XLanes& xl, bool prev_in, bool next_in, unsigned from_prev,
                                              unsigned from_next) {
  unsigned short* u = reinterpret_cast<unsigned short*>(p);
  if (cx == 0) {
    *reinterpret_cast<uint2*>(p + i0) = Y;
  } else if (cx > 0) {  // cell i0+m -> element i0+m+1
    unsigned prev = __shfl_sync(0xffffffffu, Y.y >> 16, xl.src_prev);  // cell i0-1 of the lane before
    if (xl.edge_prev && prev_in) prev = from_prev;
    const unsigned lo = __byte_perm(prev, Y.x, 0x5410), hi = __byte_perm(Y.x, Y.y, 0x5432);
    if (!xl.edge_prev || prev_in) {
      *reinterpret_cast<uint2*>(p + i0) = make_uint2(lo, hi);
    } else {
      u[i0 + 1] = (unsigned short)(Y.x & 0xffffu);
      *reinterpret_cast<unsigned*>(p + i0 + 2) = hi;
    }
    if (xl.edge_next && !next_in) u[i_next] = (unsigned short)(Y.y >> 16);
  } else {  // cell i0+m -> element i0+m-1
    unsigned next = __shfl_sync(0xffffffffu, Y.x & 0xffffu, xl.src_next);  // cell i0+4 of the lane after
    if (xl.edge_next && next_in) next = from_next;
    const unsigned lo = __byte_perm(Y.x, Y.y, 0x5432), hi = __byte_perm(Y.y, next, 0x5432);
    if (!xl.edge_next || next_in) {
      *reinterpret_cast<uint2*>(p + i0) = make_uint2(lo, hi);
    } else {
      *reinterpret_cast<unsigned*>(p + i0) = lo;
      u[i0 + 2] = (unsigned short)(Y.y >> 16);
    }
    if (xl.edge_prev && !prev_in) u[i_prev] = (unsigned short)(Y.x & 0xffffu);
  }
}

template <bool ODD, bool LES>
__global__ void __launch_bounds__(128, 5) k_aa_f16v(Pops<__half> a, Geo g, StepK K, int log_tpr) {
  const int tpr = 1 << log_tpr;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int j0 = t >> log_tpr, pos = t & (tpr - 1);
  const int k = blockIdx.y;
  const bool valid = j0 < g.ny;  // whole warps: ny*tpr is a multiple of 32
  if (!ODD && !valid) return;
  const int j = valid ? j0 : 0;  // an idle warp of the odd step only reaches its barrier
  const XLanes xl(tpr, pos, threadIdx.x & 31);
  const int i0 = pos * 4;
  const int jm = j == 0 ? g.ny - 1 : j - 1, jp = j == g.ny - 1 ? 0 : j + 1;
  const int km = k == 0 ? g.nz - 1 : k - 1, kp = k == g.nz - 1 ? 0 : k + 1;
  const int i_prev = pos == 0 ? g.nx - 1 : i0 - 1;
  const int i_next = pos == tpr - 1 ? 0 : i0 + 4;
  auto row = [&](int dy, int dz) {  // row offset of (j + dy, k + dz), dy, dz in {-1, 0, 1}
    const int jj = dy > 0 ? jp : (dy < 0 ? jm : j);
    const int kk = dz > 0 ? kp : (dz < 0 ? km : k);
    return g.sx * (jj + g.ny * kk);
  };
  uint2 Y[Q];
  if (ODD && !valid) {
#pragma unroll
    for (int q = 0; q < Q; ++q) Y[q] = make_uint2(0u, 0u);
  } else if (ODD) {
    unsigned short E[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const __half* p = a.p[oppq(q)] + row(-cyq(q), -czq(q));
      Y[q] = __ldg(reinterpret_cast<const uint2*>(p + i0));
      E[q] = 0;
      if (cxq(q) > 0 && xl.edge_prev) E[q] = ldg_u16(p + i_prev);
      if (cxq(q) < 0 && xl.edge_next) E[q] = ldg_u16(p + i_next);
    }
    shift_rows(Y, E, xl);
  } else {
#pragma unroll
    for (int q = 0; q < Q; ++q) Y[q] = __ldg(reinterpret_cast<const uint2*>(a.p[q] + row(0, 0) + i0));
  }
  if (valid) collide4_f16<LES>(Y, K);
  // odd step: the warps' crossing values (cx > 0 populations: the last
  // lane's last cell; cx < 0: the first lane's first cell) through shared
  // memory; the barrier also orders every warp's loads before any warp's
  // stores of its neighbours' crossing elements
  __shared__ unsigned xs_last[ODD ? 4 : 1][5], xs_first[ODD ? 4 : 1][5];
  bool prev_in = false, next_in = false;
  int wprev = 0, wnext = 0;
  if (ODD) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (tpr >= 32) {
      const int nw = tpr >> 5, r = pos >> 5;  // warps per row, this warp's place in its row
      if (nw <= 4) {  // the whole row in this block
        prev_in = next_in = true;
        wprev = w - r + (r + nw - 1) % nw;
        wnext = w - r + (r + 1) % nw;
      } else {
        prev_in = w > 0;
        next_in = w < 3;
        wprev = w - 1;
        wnext = w + 1;
      }
      if (valid && lane == 31) {
#pragma unroll
        for (int q = 0; q < 5; ++q) xs_last[w][q] = Y[q].y >> 16;
      }
      if (valid && lane == 0) {
#pragma unroll
        for (int q = 9; q < 14; ++q) xs_first[w][q - 9] = Y[q].x & 0xffffu;
      }
    }
    __syncthreads();
    if (!valid) return;
  }
  int js = j, ks = k;  // store rows: recomputed after the collision (BGK odd step)
  if (ODD) asm volatile("" : "+r"(js), "+r"(ks));
  const int jms = js == 0 ? g.ny - 1 : js - 1, jps = js == g.ny - 1 ? 0 : js + 1;
  const int kms = ks == 0 ? g.nz - 1 : ks - 1, kps = ks == g.nz - 1 ? 0 : ks + 1;
  auto row_out = [&](int dy, int dz) {
    const int jj = dy > 0 ? jps : (dy < 0 ? jms : js);
    const int kk = dz > 0 ? kps : (dz < 0 ? kms : ks);
    return g.sx * (jj + g.ny * kk);
  };
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    if (!ODD) {
      *reinterpret_cast<uint2*>(a.p[oppq(q)] + row(0, 0) + i0) = Y[q];
    } else {
      const unsigned fp = cxq(q) > 0 && xl.edge_prev && prev_in ? xs_last[wprev][q] : 0u;
      const unsigned fn = cxq(q) < 0 && xl.edge_next && next_in ? xs_first[wnext][q - 9] : 0u;
      shift_out(Y[q], cxq(q), a.p[q] + row_out(cyq(q), czq(q)), i0, i_prev, i_next, xl, prev_in, next_in, fp, fn);
    }
  }
}

// FP16 AA pattern with eight cells per thread: k_aa_f16v's structure on
// 16-byte chunks (cells i0..i0+7, i0 = 8 pos, tpr = nx/8 threads per row), so
// the per-thread work of the odd step's x-crossing (shuffles, warp-edge
// values, the 18 shifted rows' addresses) is spread over twice the cells.
// Per-cell arithmetic is collide4_f16's on each half of the chunk, so the
// results are k_aa_f16v's. The odd instantiation is launched (128
// registers, 4 blocks/SM); the even one measured no faster than k_aa_f16v.
__device__ __forceinline__ void shift_rows8(uint4 (&Y)[Q], const unsigned short (&E)[Q], const XLanes& xl) {
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const uint4 A = Y[q];
    if (cxq(q) > 0) {  // elements i0-1 .. i0+6
      unsigned prev = __shfl_sync(0xffffffffu, A.w >> 16, xl.src_prev);
      if (xl.edge_prev) prev = E[q];
      Y[q].x = __byte_perm(A.x, prev, 0x1054);
      Y[q].y = __byte_perm(A.x, A.y, 0x5432);
      Y[q].z = __byte_perm(A.y, A.z, 0x5432);
      Y[q].w = __byte_perm(A.z, A.w, 0x5432);
    } else if (cxq(q) < 0) {  // elements i0+1 .. i0+8
      unsigned next = __shfl_sync(0xffffffffu, A.x & 0xffffu, xl.src_next);
      if (xl.edge_next) next = E[q];
      Y[q].x = __byte_perm(A.x, A.y, 0x5432);
      Y[q].y = __byte_perm(A.y, A.z, 0x5432);
      Y[q].z = __byte_perm(A.z, A.w, 0x5432);
      Y[q].w = __byte_perm(A.w, next, 0x5432);
    }
  }
}

// Store side of the eight-cells odd step (shift_out on 16-byte chunks): cell
// i0+m goes to element i0+m+cx; the aligned chunk i0..i0+7 is completed with
// the neighbouring lane's crossing value, and at block boundaries the edge
// lanes store their part with 2-, 4- and 8-byte stores.
__device__ __forceinline__ void shift_out8(uint4 Y, int cx, __half* p, int i0, int i_prev, int i_next,
                                           const XLanes& xl, bool prev_in, bool next_in, unsigned from_prev,
                                           unsigned from_next) {
  unsigned short* u = reinterpret_cast<unsigned short*>(p);
  if (cx == 0) {
    *reinterpret_cast<uint4*>(p + i0) = Y;
  } else if (cx > 0) {  // cell i0+m -> element i0+m+1
    unsigned prev = __shfl_sync(0xffffffffu, Y.w >> 16, xl.src_prev);  // cell i0-1 of the lane before
    if (xl.edge_prev && prev_in) prev = from_prev;
    const uint4 c = make_uint4(__byte_perm(prev, Y.x, 0x5410), __byte_perm(Y.x, Y.y, 0x5432),
                               __byte_perm(Y.y, Y.z, 0x5432), __byte_perm(Y.z, Y.w, 0x5432));
    if (!xl.edge_prev || prev_in) {
      *reinterpret_cast<uint4*>(p + i0) = c;
    } else {
      u[i0 + 1] = (unsigned short)(Y.x & 0xffffu);
      *reinterpret_cast<unsigned*>(p + i0 + 2) = c.y;
      *reinterpret_cast<uint2*>(p + i0 + 4) = make_uint2(c.z, c.w);
    }
    if (xl.edge_next && !next_in) u[i_next] = (unsigned short)(Y.w >> 16);
  } else {  // cell i0+m -> element i0+m-1
    unsigned next = __shfl_sync(0xffffffffu, Y.x & 0xffffu, xl.src_next);  // cell i0+8 of the lane after
    if (xl.edge_next && next_in) next = from_next;
    const uint4 c = make_uint4(__byte_perm(Y.x, Y.y, 0x5432), __byte_perm(Y.y, Y.z, 0x5432),
                               __byte_perm(Y.z, Y.w, 0x5432), __byte_perm(Y.w, next, 0x5432));
    if (!xl.edge_next || next_in) {
      *reinterpret_cast<uint4*>(p + i0) = c;
    } else {
      *reinterpret_cast<uint2*>(p + i0) = make_uint2(c.x, c.y);
      *reinterpret_cast<unsigned*>(p + i0 + 4) = c.z;
      u[i0 + 6] = (unsigned short)(Y.w >> 16);
    }
    if (xl.edge_prev && !prev_in) u[i_prev] = (unsigned short)(Y.x & 0xffffu);
  }
}

template <bool ODD>
__global__ void __launch_bounds__(128, 4) k_aa_f16w(Pops<__half> a, Geo g, StepK K, int log_tpr) {
  const int tpr = 1 << log_tpr;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int j0 = t >> log_tpr, pos = t & (tpr - 1);
  const int k = blockIdx.y;
  const bool valid = j0 < g.ny;  // whole warps: ny*tpr is a multiple of 32
  if (!ODD && !valid) return;
  const int j = valid ? j0 : 0;  // an idle warp of the odd step only reaches its barrier
  const XLanes xl(tpr, pos, threadIdx.x & 31);
  const int i0 = pos * 8;
  const int jm = j == 0 ? g.ny - 1 : j - 1, jp = j == g.ny - 1 ? 0 : j + 1;
  const int km = k == 0 ? g.nz - 1 : k - 1, kp = k == g.nz - 1 ? 0 : k + 1;
  const int i_prev = pos == 0 ? g.nx - 1 : i0 - 1;
  const int i_next = pos == tpr - 1 ? 0 : i0 + 8;
  auto row = [&](int dy, int dz) {
    const int jj = dy > 0 ? jp : (dy < 0 ? jm : j);
    const int kk = dz > 0 ? kp : (dz < 0 ? km : k);
    return g.sx * (jj + g.ny * kk);
  };
  uint4 Y[Q];
  if (ODD && !valid) {
#pragma unroll
    for (int q = 0; q < Q; ++q) Y[q] = make_uint4(0u, 0u, 0u, 0u);
  } else if (ODD) {
    unsigned short E[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const __half* p = a.p[oppq(q)] + row(-cyq(q), -czq(q));
      Y[q] = __ldg(reinterpret_cast<const uint4*>(p + i0));
      E[q] = 0;
      if (cxq(q) > 0 && xl.edge_prev) E[q] = ldg_u16(p + i_prev);
      if (cxq(q) < 0 && xl.edge_next) E[q] = ldg_u16(p + i_next);
    }
    shift_rows8(Y, E, xl);
  } else {
#pragma unroll
    for (int q = 0; q < Q; ++q) Y[q] = __ldg(reinterpret_cast<const uint4*>(a.p[q] + row(0, 0) + i0));
  }
  if (valid) {
    uint2 L[Q], H[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      L[q] = make_uint2(Y[q].x, Y[q].y);
      H[q] = make_uint2(Y[q].z, Y[q].w);
    }
    collide4_f16<false>(L, K);
    collide4_f16<false>(H, K);
#pragma unroll
    for (int q = 0; q < Q; ++q) Y[q] = make_uint4(L[q].x, L[q].y, H[q].x, H[q].y);
  }
  __shared__ unsigned xs_last[ODD ? 4 : 1][5], xs_first[ODD ? 4 : 1][5];
  bool prev_in = false, next_in = false;
  int wprev = 0, wnext = 0;
  if (ODD) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (tpr >= 32) {
      const int nw = tpr >> 5, r = pos >> 5;
      if (nw <= 4) {
        prev_in = next_in = true;
        wprev = w - r + (r + nw - 1) % nw;
        wnext = w - r + (r + 1) % nw;
      } else {
        prev_in = w > 0;
        next_in = w < 3;
        wprev = w - 1;
        wnext = w + 1;
      }
      if (valid && lane == 31) {
#pragma unroll
        for (int q = 0; q < 5; ++q) xs_last[w][q] = Y[q].w >> 16;
      }
      if (valid && lane == 0) {
#pragma unroll
        for (int q = 9; q < 14; ++q) xs_first[w][q - 9] = Y[q].x & 0xffffu;
      }
    }
    __syncthreads();
    if (!valid) return;
  }
  int js = j, ks = k;
  if (ODD) asm volatile("" : "+r"(js), "+r"(ks));
  const int jms = js == 0 ? g.ny - 1 : js - 1, jps = js == g.ny - 1 ? 0 : js + 1;
  const int kms = ks == 0 ? g.nz - 1 : ks - 1, kps = ks == g.nz - 1 ? 0 : ks + 1;
  auto row_out = [&](int dy, int dz) {
    const int jj = dy > 0 ? jps : (dy < 0 ? jms : js);
    const int kk = dz > 0 ? kps : (dz < 0 ? kms : ks);
    return g.sx * (jj + g.ny * kk);
  };
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    if (!ODD) {
      *reinterpret_cast<uint4*>(a.p[oppq(q)] + row(0, 0) + i0) = Y[q];
    } else {
      const unsigned fp = cxq(q) > 0 && xl.edge_prev && prev_in ? xs_last[wprev][q] : 0u;
      const unsigned fn = cxq(q) < 0 && xl.edge_next && next_in ? xs_first[wnext][q - 9] : 0u;
      shift_out8(Y[q], cxq(q), a.p[q] + row_out(cyq(q), czq(q)), i0, i_prev, i_next, xl, prev_in, next_in, fp, fn);
    }
  }
}

// Store side of the FP32 odd step: cells i0, i0+1 go to elements i0 + cx,
// i0 + 1 + cx of row p, stored as the aligned chunk (i0, i0+1) completed with
// the neighbouring lane's crossing value, as shift_out does for FP16.
__device__ __forceinline__ void shift_out_f32(float2 Y, int cx, float* p, int i0, int i_prev, int i_next,
                                              const XLanes& xl, bool prev_in, bool next_in, float from_prev,
                                              float from_next) {
  if (cx == 0) {
    *reinterpret_cast<float2*>(p + i0) = Y;
  } else if (cx > 0) {  // cell i0+m -> element i0+m+1
    float prev = __shfl_sync(0xffffffffu, Y.y, xl.src_prev);  // cell i0-1 of the lane before
    if (xl.edge_prev && prev_in) prev = from_prev;
    if (!xl.edge_prev || prev_in) *reinterpret_cast<float2*>(p + i0) = make_float2(prev, Y.x);
    else p[i0 + 1] = Y.x;
    if (xl.edge_next && !next_in) p[i_next] = Y.y;
  } else {  // cell i0+m -> element i0+m-1
    float next = __shfl_sync(0xffffffffu, Y.x, xl.src_next);  // cell i0+2 of the lane after
    if (xl.edge_next && next_in) next = from_next;
    if (!xl.edge_next || next_in) *reinterpret_cast<float2*>(p + i0) = make_float2(Y.y, next);
    else p[i0] = Y.y;
    if (xl.edge_prev && !prev_in) p[i_prev] = Y.x;
  }
}

// FP32 AA pattern with two cells per thread: k_aa_f16v's row split (tpr =
// nx/2 threads per row), x-crossing shuffles and block-local warp-edge stores
// on 8-byte chunks of two floats, F32::cell's arithmetic (the reference's
// order) on each cell, so the results are those of k_aa<F32, ODD>. The same
// ownership argument keeps the in-place update race-free. 95 registers (87
// for the Smagorinsky even step), no spills.
template <bool ODD, bool LES>
__global__ void __launch_bounds__(128, 5) k_aa_f32v(Pops<float> a, Geo g, StepK K, int log_tpr) {
  const int tpr = 1 << log_tpr;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int j0 = t >> log_tpr, pos = t & (tpr - 1);
  const int k = blockIdx.y;
  const bool valid = j0 < g.ny;  // whole warps: ny*tpr is a multiple of 32
  if (!ODD && !valid) return;
  const int j = valid ? j0 : 0;  // an idle warp of the odd step only reaches its barrier
  const XLanes xl(tpr, pos, threadIdx.x & 31);
  const int i0 = pos * 2;
  const int jm = j == 0 ? g.ny - 1 : j - 1, jp = j == g.ny - 1 ? 0 : j + 1;
  const int km = k == 0 ? g.nz - 1 : k - 1, kp = k == g.nz - 1 ? 0 : k + 1;
  const int i_prev = pos == 0 ? g.nx - 1 : i0 - 1;
  const int i_next = pos == tpr - 1 ? 0 : i0 + 2;
  auto row = [&](int dy, int dz) {  // row offset of (j + dy, k + dz), dy, dz in {-1, 0, 1}
    const int jj = dy > 0 ? jp : (dy < 0 ? jm : j);
    const int kk = dz > 0 ? kp : (dz < 0 ? km : k);
    return g.sx * (jj + g.ny * kk);
  };
  float2 Y[Q];
  if (ODD && !valid) {
#pragma unroll
    for (int q = 0; q < Q; ++q) Y[q] = make_float2(0.f, 0.f);
  } else if (ODD) {
    float E[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const float* p = a.p[oppq(q)] + row(-cyq(q), -czq(q));
      Y[q] = __ldg(reinterpret_cast<const float2*>(p + i0));
      E[q] = 0.f;
      if (cxq(q) > 0 && xl.edge_prev) E[q] = __ldg(p + i_prev);
      if (cxq(q) < 0 && xl.edge_next) E[q] = __ldg(p + i_next);
    }
    shift_rows_f32(Y, E, xl);
  } else {
#pragma unroll
    for (int q = 0; q < Q; ++q) Y[q] = __ldg(reinterpret_cast<const float2*>(a.p[q] + row(0, 0) + i0));
  }
  if (valid) {
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      float s[Q];
#pragma unroll
      for (int q = 0; q < Q; ++q) s[q] = m ? Y[q].y : Y[q].x;
      F32::cell<LES>(s, K);
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        if (m) Y[q].y = s[q];
        else Y[q].x = s[q];
      }
    }
  }
  __shared__ float xs_last[ODD ? 4 : 1][5], xs_first[ODD ? 4 : 1][5];
  bool prev_in = false, next_in = false;
  int wprev = 0, wnext = 0;
  if (ODD) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (tpr >= 32) {
      const int nw = tpr >> 5, r = pos >> 5;  // warps per row, this warp's place in its row
      if (nw <= 4) {  // the whole row in this block
        prev_in = next_in = true;
        wprev = w - r + (r + nw - 1) % nw;
        wnext = w - r + (r + 1) % nw;
      } else {
        prev_in = w > 0;
        next_in = w < 3;
        wprev = w - 1;
        wnext = w + 1;
      }
      if (valid && lane == 31) {
#pragma unroll
        for (int q = 0; q < 5; ++q) xs_last[w][q] = Y[q].y;
      }
      if (valid && lane == 0) {
#pragma unroll
        for (int q = 9; q < 14; ++q) xs_first[w][q - 9] = Y[q].x;
      }
    }
    __syncthreads();
    if (!valid) return;
  }
  int js = j, ks = k;  // store rows: recomputed after the collision
  if (ODD) asm volatile("" : "+r"(js), "+r"(ks));
  const int jms = js == 0 ? g.ny - 1 : js - 1, jps = js == g.ny - 1 ? 0 : js + 1;
  const int kms = ks == 0 ? g.nz - 1 : ks - 1, kps = ks == g.nz - 1 ? 0 : ks + 1;
  auto row_out = [&](int dy, int dz) {
    const int jj = dy > 0 ? jps : (dy < 0 ? jms : js);
    const int kk = dz > 0 ? kps : (dz < 0 ? kms : ks);
    return g.sx * (jj + g.ny * kk);
  };
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    if (!ODD) {
      *reinterpret_cast<float2*>(a.p[oppq(q)] + row(0, 0) + i0) = Y[q];
    } else {
      const float fp = cxq(q) > 0 && xl.edge_prev && prev_in ? xs_last[wprev][q] : 0.f;
      const float fn = cxq(q) < 0 && xl.edge_next && next_in ? xs_first[wnext][q - 9] : 0.f;
      shift_out_f32(Y[q], cxq(q), a.p[q] + row_out(cyq(q), czq(q)), i0, i_prev, i_next, xl, prev_in, next_in, fp,
                    fn);
    }
  }
}

// FP32 AA odd step with four cells per thread: k_aa_f32v's odd step on
// 16-byte chunks of four floats (cells i0..i0+3, i0 = 4 pos, tpr = nx/4), so
// its per-thread x-crossing work covers twice the cells, as k_aa_f16w does
// for FP16. F32::cell's arithmetic on each cell: the results of k_aa<F32>.
// 125 registers (127 with the Smagorinsky collision), 4 blocks/SM, no spills.
__device__ __forceinline__ void shift_out4_f32(float4 Y, int cx, float* p, int i0, int i_prev, int i_next,
                                               const XLanes& xl, bool prev_in, bool next_in, float from_prev,
                                               float from_next) {
  if (cx == 0) {
    *reinterpret_cast<float4*>(p + i0) = Y;
  } else if (cx > 0) {  // cell i0+m -> element i0+m+1
    float prev = __shfl_sync(0xffffffffu, Y.w, xl.src_prev);  // cell i0-1 of the lane before
    if (xl.edge_prev && prev_in) prev = from_prev;
    if (!xl.edge_prev || prev_in) {
      *reinterpret_cast<float4*>(p + i0) = make_float4(prev, Y.x, Y.y, Y.z);
    } else {
      p[i0 + 1] = Y.x;
      *reinterpret_cast<float2*>(p + i0 + 2) = make_float2(Y.y, Y.z);
    }
    if (xl.edge_next && !next_in) p[i_next] = Y.w;
  } else {  // cell i0+m -> element i0+m-1
    float next = __shfl_sync(0xffffffffu, Y.x, xl.src_next);  // cell i0+4 of the lane after
    if (xl.edge_next && next_in) next = from_next;
    if (!xl.edge_next || next_in) {
      *reinterpret_cast<float4*>(p + i0) = make_float4(Y.y, Y.z, Y.w, next);
    } else {
      *reinterpret_cast<float2*>(p + i0) = make_float2(Y.y, Y.z);
      p[i0 + 2] = Y.w;
    }
    if (xl.edge_prev && !prev_in) p[i_prev] = Y.x;
  }
}

template <bool LES = false>
__global__ void __launch_bounds__(128, 4) k_aa_f32w(Pops<float> a, Geo g, StepK K, int log_tpr) {
  const int tpr = 1 << log_tpr;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int j0 = t >> log_tpr, pos = t & (tpr - 1);
  const int k = blockIdx.y;
  const bool valid = j0 < g.ny;  // whole warps: ny*tpr is a multiple of 32
  const int j = valid ? j0 : 0;  // an idle warp only reaches its barrier
  const XLanes xl(tpr, pos, threadIdx.x & 31);
  const int i0 = pos * 4;
  const int jm = j == 0 ? g.ny - 1 : j - 1, jp = j == g.ny - 1 ? 0 : j + 1;
  const int km = k == 0 ? g.nz - 1 : k - 1, kp = k == g.nz - 1 ? 0 : k + 1;
  const int i_prev = pos == 0 ? g.nx - 1 : i0 - 1;
  const int i_next = pos == tpr - 1 ? 0 : i0 + 4;
  auto row = [&](int dy, int dz) {
    const int jj = dy > 0 ? jp : (dy < 0 ? jm : j);
    const int kk = dz > 0 ? kp : (dz < 0 ? km : k);
    return g.sx * (jj + g.ny * kk);
  };
  float4 Y[Q];
  if (!valid) {
#pragma unroll
    for (int q = 0; q < Q; ++q) Y[q] = make_float4(0.f, 0.f, 0.f, 0.f);
  } else {
    float E[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const float* p = a.p[oppq(q)] + row(-cyq(q), -czq(q));
      Y[q] = __ldg(reinterpret_cast<const float4*>(p + i0));
      E[q] = 0.f;
      if (cxq(q) > 0 && xl.edge_prev) E[q] = __ldg(p + i_prev);
      if (cxq(q) < 0 && xl.edge_next) E[q] = __ldg(p + i_next);
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const float4 A = Y[q];
      if (cxq(q) > 0) {  // elements i0-1 .. i0+2
        float prev = __shfl_sync(0xffffffffu, A.w, xl.src_prev);
        if (xl.edge_prev) prev = E[q];
        Y[q] = make_float4(prev, A.x, A.y, A.z);
      } else if (cxq(q) < 0) {  // elements i0+1 .. i0+4
        float next = __shfl_sync(0xffffffffu, A.x, xl.src_next);
        if (xl.edge_next) next = E[q];
        Y[q] = make_float4(A.y, A.z, A.w, next);
      }
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      float s[Q];
#pragma unroll
      for (int q = 0; q < Q; ++q) s[q] = m == 0 ? Y[q].x : (m == 1 ? Y[q].y : (m == 2 ? Y[q].z : Y[q].w));
      F32::cell<LES>(s, K);
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        if (m == 0) Y[q].x = s[q];
        else if (m == 1) Y[q].y = s[q];
        else if (m == 2) Y[q].z = s[q];
        else Y[q].w = s[q];
      }
    }
  }
  __shared__ float xs_last[4][5], xs_first[4][5];
  bool prev_in = false, next_in = false;
  int wprev = 0, wnext = 0;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (tpr >= 32) {
    const int nw = tpr >> 5, r = pos >> 5;  // warps per row, this warp's place in its row
    if (nw <= 4) {  // the whole row in this block
      prev_in = next_in = true;
      wprev = w - r + (r + nw - 1) % nw;
      wnext = w - r + (r + 1) % nw;
    } else {
      prev_in = w > 0;
      next_in = w < 3;
      wprev = w - 1;
      wnext = w + 1;
    }
    if (valid && lane == 31) {
#pragma unroll
      for (int q = 0; q < 5; ++q) xs_last[w][q] = Y[q].w;
    }
    if (valid && lane == 0) {
#pragma unroll
      for (int q = 9; q < 14; ++q) xs_first[w][q - 9] = Y[q].x;
    }
  }
  __syncthreads();
  if (!valid) return;
  int js = j, ks = k;  // store rows: recomputed after the collision
  asm volatile("" : "+r"(js), "+r"(ks));
  const int jms = js == 0 ? g.ny - 1 : js - 1, jps = js == g.ny - 1 ? 0 : js + 1;
  const int kms = ks == 0 ? g.nz - 1 : ks - 1, kps = ks == g.nz - 1 ? 0 : ks + 1;
  auto row_out = [&](int dy, int dz) {
    const int jj = dy > 0 ? jps : (dy < 0 ? jms : js);
    const int kk = dz > 0 ? kps : (dz < 0 ? kms : ks);
    return g.sx * (jj + g.ny * kk);
  };
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const float fp = cxq(q) > 0 && xl.edge_prev && prev_in ? xs_last[wprev][q] : 0.f;
    const float fn = cxq(q) < 0 && xl.edge_next && next_in ? xs_first[wnext][q - 9] : 0.f;
    shift_out4_f32(Y[q], cxq(q), a.p[q] + row_out(cyq(q), czq(q)), i0, i_prev, i_next, xl, prev_in, next_in, fp, fn);
  }
}

// ----------------------------------------------------------------- z-slabs
// Two-lattice step of one z-slab of a box split along z (the reference's
// proc_z ranks, SRC/setup_MPI.F90:112-131). x and y wrap in the kernel; a pull
// across a z face reads this slab's ghost plane instead of wrapping. The
// boundary planes' post-collision populations that cross a face are also
// stored straight into the neighbour's ghost plane for the next step (a peer
// store over NVLink when the neighbour is another GPU): the halo exchange of
// SRC/bcond.comm.step3.F90:77-297 fused into the producing kernel.
// EDGE = false: the interior planes 1..nz-2 (blockIdx.z + 1), whose pulls stay
// inside the slab (the whole-box kernel's code without the z wrap); EDGE =
// true: planes 0 and nz-1 (blockIdx.z = 0, 1), which read ghost planes and
// feed the neighbours. Separate kernels keep the interior one's registers
// (and so its occupancy) those of the whole-box kernel.
template <class F, bool LES, bool EDGE>
__global__ void __launch_bounds__(256) k_slab(Pops<const typename F::S> src, Pops<typename F::S> dst, Geo g,
                                              StepK K, Halo<typename F::S> h) {
  using S = typename F::S;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = EDGE ? (blockIdx.z == 0 ? 0 : g.nz - 1) : (int)blockIdx.z + 1;
  const bool active = i < g.nx && j < g.ny;
  if (!EDGE && !active) return;
  if (active) {
    const int im = i == 0 ? g.nx - 1 : i - 1, ip = i == g.nx - 1 ? 0 : i + 1;
    const int jm = j == 0 ? g.ny - 1 : j - 1, jp = j == g.ny - 1 ? 0 : j + 1;
    S v[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int ii = cxq(q) > 0 ? im : (cxq(q) < 0 ? ip : i);
      const int jj = cyq(q) > 0 ? jm : (cyq(q) < 0 ? jp : j);
      const int po = ii + g.sx * jj;
      if (EDGE && czq(q) > 0 && k == 0) v[q] = ldg(h.in_lo[zslot(q)] + po);
      else if (EDGE && czq(q) < 0 && k == g.nz - 1) v[q] = ldg(h.in_hi[zslot(q)] + po);
      else {
        const int off = po + g.sx * g.ny * (k - czq(q));
        v[q] = (q == Q - 1) ? src.p[Q - 1][off] : ldg(src.p[q] + off);
      }
    }
    F::template cell<LES>(v, K);
    const int po = i + g.sx * j;
    const int o = po + g.sx * g.ny * k;
#pragma unroll
    for (int q = 0; q < Q; ++q) dst.p[q][o] = v[q];
    if (EDGE && k == g.nz - 1) {
#pragma unroll
      for (int q = 0; q < Q; ++q)
        if (czq(q) > 0) h.up[zslot(q)][po] = v[q];
    }
    if (EDGE && k == 0) {
#pragma unroll
      for (int q = 0; q < Q; ++q)
        if (czq(q) < 0) h.dn[zslot(q)][po] = v[q];
    }
  }
  if (EDGE) {
    // the block's stores into the neighbour's planes (peer memory when the
    // neighbour is another GPU) are made visible system-wide before the
    // kernel ends: a block barrier, then one system-scope fence (cumulative
    // over the stores the barrier ordered before it)
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) __threadfence_system();
  }
}

// Fills the neighbours' ghost planes from this slab's current boundary planes
// (after an initial condition, an upload or a restart).
template <class S>
__global__ void k_halo_prime(Pops<const S> a, Geo g, Halo<S> h) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i < g.nx) {
    const int po = i + g.sx * j;
    const long long top = po + (long long)g.sx * g.ny * (g.nz - 1);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if (czq(q) > 0) h.up[zslot(q)][po] = a.p[q][top];
      if (czq(q) < 0) h.dn[zslot(q)][po] = a.p[q][po];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) __threadfence_system();
}

// ------------------------------------------------------ initial conditions
// Per-cell equilibrium deviation of SRC/init.F90:97-137 (cte1 = 0):
// out_q = crho*w_q*(0 + rf*(c.u) + qf*(3*(c.u)^2 - |u|^2)), with each linear
// and quadratic term written as in the reference text.
template <class V>
__device__ __forceinline__ void eq_init(V xj, V yj, V zj, V crho, V (&out)[Q]) {
  using N = Num<V>;
  const V rf = N::c(3.0), qf = N::c(1.5), three = N::c(3.0), zero = N::c(0.0), cte1 = zero;
  const V p0 = N::c(1.0 / 3.0), p1 = N::c(1.0 / 18.0), p2 = N::c(1.0 / (3.0 * 3.0 * (1.0 + 3.0)));
  const V cvsq = xj * xj + yj * yj + zj * zj;
  V cx[Q];
  cx[0]  = rf * (xj - yj) + qf * (three * (xj - yj) * (xj - yj) - cvsq);
  cx[1]  = rf * (xj - zj) + qf * (three * (xj - zj) * (xj - zj) - cvsq);
  cx[2]  = rf * (xj + yj) + qf * (three * (xj + yj) * (xj + yj) - cvsq);
  cx[3]  = rf * (xj + zj) + qf * (three * (xj + zj) * (xj + zj) - cvsq);
  cx[4]  = rf * (xj) + qf * (three * (xj) * (xj) - cvsq);
  cx[5]  = rf * (zj) + qf * (three * (zj) * (zj) - cvsq);
  cx[6]  = rf * (yj + zj) + qf * (three * (yj + zj) * (yj + zj) - cvsq);
  cx[7]  = rf * (yj) + qf * (three * (yj) * (yj) - cvsq);
  cx[8]  = rf * (yj - zj) + qf * (three * (yj - zj) * (yj - zj) - cvsq);
  cx[9]  = rf * (-xj - yj) + qf * (three * (xj + yj) * (xj + yj) - cvsq);
  cx[10] = rf * (-xj - zj) + qf * (three * (xj + zj) * (xj + zj) - cvsq);
  cx[11] = rf * (-xj + yj) + qf * (three * (xj - yj) * (xj - yj) - cvsq);
  cx[12] = rf * (-xj + zj) + qf * (three * (xj - zj) * (xj - zj) - cvsq);
  cx[13] = rf * (-xj) + qf * (three * (xj) * (xj) - cvsq);
  cx[14] = rf * (-zj) + qf * (three * (zj) * (zj) - cvsq);
  cx[15] = rf * (-yj - zj) + qf * (three * (yj + zj) * (yj + zj) - cvsq);
  cx[16] = rf * (-yj) + qf * (three * (yj) * (yj) - cvsq);
  cx[17] = rf * (-yj + zj) + qf * (three * (yj - zj) * (yj - zj) - cvsq);
  cx[18] = rf * zero + qf * (three * zero * zero - cvsq);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const bool w1 = (q == 4 || q == 5 || q == 7 || q == 13 || q == 14 || q == 16);
    const V w = q == 18 ? p0 : (w1 ? p1 : p2);
    out[q] = crho * w * (cte1 + cx[q]);
  }
}

__device__ __forceinline__ double dsin(double x) { return sin(x); }
__device__ __forceinline__ double dcos(double x) { return cos(x); }
__device__ __forceinline__ float dsin(float x) { return sinf(x); }
__device__ __forceinline__ float dcos(float x) { return cosf(x); }

template <class F>
__device__ __forceinline__ void store_cell(Pops<typename F::S>& a, int lay, int o, typename F::V (&v)[Q],
                                           typename F::R scale) {
  using N = Num<typename F::V>;
#pragma unroll
  for (int q = 0; q < Q; ++q) a.p[lay == LAY_AAE ? oppq(q) : q][o] = F::enc(N::raw(v[q]), scale);
}

// Largest |deviation| of a cell, for choosing the FP16 scale.
template <class V>
__device__ __forceinline__ float cell_maxabs(const V (&v)[Q]) {
  float m = 0.f;
#pragma unroll
  for (int q = 0; q < Q; ++q) m = fmaxf(m, fabsf((float)Num<V>::raw(v[q])));
  return m;
}

// Taylor-Green vortex, SRC/init.F90:83-141 (offsets zero, one box).
// maxbits != nullptr: measure max |deviation| only (atomicMax on the bits of a
// non-negative float), store nothing.
template <class F>
__global__ void k_init_tgv(Pops<typename F::S> a, Geo g, int lay, typename F::R u0r, int faithful,
                           typename F::R scale, unsigned int* maxbits) {
  using R = typename F::R; using V = typename F::V; using N = Num<V>;
  const long long n = (long long)g.nx * g.ny * g.nz;
  float tmax = 0.f;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long long)g.nx * g.ny));
    // reference interior indices are 1-based; a z-slab uses global z
    // (k0 + k with k0 = offset(3), SRC/init.F90:73,84)
    const int ir = i + 1, jr = j + 1, kr = g.z0 + k + 1;
    const int gz = g.gz > 0 ? g.gz : g.nz;
    R x, y, z, pi;
    if (faithful) {
      x = (R)(((float)ir - 0.5f) / (float)g.nx);
      y = (R)(((float)jr - 0.5f) / (float)g.ny);
      z = (R)(((float)kr - 0.5f) / (float)gz);
      pi = (R)3.141592653589793238462643383279f;
    } else {
      x = (R)(((double)ir - 0.5) / (double)g.nx);
      y = (R)(((double)jr - 0.5) / (double)g.ny);
      z = (R)(((double)kr - 0.5) / (double)gz);
      pi = (R)3.141592653589793238462643383279;
    }
    const V two = N::c(2.0), four = N::c(4.0), u0 = N::wrap(u0r), P = N::wrap(pi);
    const V X = N::wrap(x), Y = N::wrap(y), Z = N::wrap(z);
    const R ax = N::raw(two * P * X), ay = N::raw(two * P * Y), az = N::raw(two * P * Z);
    const V xj = u0 * N::wrap(dsin(ax)) * N::wrap(dcos(ay)) * N::wrap(dcos(az));
    const V yj = -(u0 * N::wrap(dcos(ax)) * N::wrap(dsin(ay)) * N::wrap(dcos(az)));
    const V zj = N::c(0.0);
    V crho = N::c(1.0);
    if (faithful) {
      const R bx = N::raw(four * P * X), by = N::raw(four * P * Y), bz = N::raw(four * P * Z);
      crho = N::c(1.0) + ((u0 * u0) / (N::c(16.0) * N::c(3.0))) * (N::wrap(dcos(bx)) + N::wrap(dcos(by))) *
                             (N::wrap(dcos(bz)) + N::c(2.0));
    }
    V out[Q];
    eq_init<V>(xj, yj, zj, crho, out);
    if (maxbits) tmax = fmaxf(tmax, cell_maxabs<V>(out));
    else store_cell<F>(a, lay, i + g.sx * (j + g.ny * k), out, scale);
  }
  if (maxbits) atomicMax(maxbits, __float_as_uint(tmax));
}

// Equilibrium from a staged velocity slab (planes k0 .. k0+nk-1, dense
// Fortran order) at uniform density rho.
template <class F>
__global__ void k_init_vel(Pops<typename F::S> a, Geo g, int lay, const double* __restrict__ u,
                           const double* __restrict__ v, const double* __restrict__ w, double rho, int k0, int nk,
                           typename F::R scale, unsigned int* maxbits) {
  using R = typename F::R; using V = typename F::V; using N = Num<V>;
  const long long n = (long long)g.nx * g.ny * nk;
  float tmax = 0.f;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = k0 + (int)(c / ((long long)g.nx * g.ny));
    V out[Q];
    eq_init<V>(N::wrap((R)u[c]), N::wrap((R)v[c]), N::wrap((R)w[c]), N::wrap((R)rho), out);
    if (maxbits) tmax = fmaxf(tmax, cell_maxabs<V>(out));
    else store_cell<F>(a, lay, i + g.sx * (j + g.ny * k), out, scale);
  }
  if (maxbits) atomicMax(maxbits, __float_as_uint(tmax));
}

// ------------------------------------------------------- reference access
// Location of the reference's a_q at cell (i,j,k) + d for a given layout.
template <int LAY>
__device__ __forceinline__ int ref_slot(int q) { return LAY == LAY_AAE ? oppq(q) : q; }
template <int LAY>
__device__ __forceinline__ int ref_off(const Geo& g, int q, int i, int j, int k, int dx, int dy, int dz) {
  if (LAY == LAY_AAN) { dx += cxq(q); dy += cyq(q); dz += czq(q); }
  return wrapi(i + dx, g.nx) + g.sx * (wrapi(j + dy, g.ny) + g.ny * wrapi(k + dz, g.nz));
}

template <class F, int LAY>
__global__ void k_export(Pops<const typename F::S> a, Geo g, int q, typename F::S* out_s, double* out_d,
                         typename F::R inv) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long long)g.nx * g.ny));
    const typename F::S s = a.p[ref_slot<LAY>(q)][ref_off<LAY>(g, q, i, j, k, 0, 0, 0)];
    if (out_s) out_s[c] = s;
    if (out_d) out_d[c] = (double)F::dec(s, inv);
  }
}

template <class F, int LAY>
__global__ void k_import(Pops<typename F::S> a, Geo g, int q, const typename F::S* __restrict__ in) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long long)g.nx * g.ny));
    a.p[ref_slot<LAY>(q)][ref_off<LAY>(g, q, i, j, k, 0, 0, 0)] = in[c];
  }
}

// ------------------------------------------------------------ diagnostics
// Quantities: 0 rho, 1 ux, 2 uy, 3 uz, 4 0.5|u|^2 (local populations,
// SRC/diagno.F90:96-111); 5 0.5|u|^2, 6 2*svisc*Ptotal (pulled populations,
// SRC/dissipation.F90:76-249); 7 2*nu*S:S with S = -3*omega*Pi/(2*rho);
// 8 non-finite cell count; 9 enstrophy (k_enstrophy).
// Offset of the periodic image of an out-of-box source cell (si, sj, sk) in a
// population's block of a boundary-plane snapshot: x planes (ny*nz each), then
// y planes (nx*nz), then z planes (nx*ny).
__device__ __forceinline__ long long faith_off(const Geo& g, int si, int sj, int sk) {
  const int wi = wrapi(si, g.nx), wj = wrapi(sj, g.ny), wk = wrapi(sk, g.nz);
  const long long yz = (long long)g.ny * g.nz, xz = (long long)g.nx * g.nz, xy = (long long)g.nx * g.ny;
  if (si < 0 || si >= g.nx) return (wi == 0 ? 0 : yz) + wj + (long long)g.ny * wk;
  if (sj < 0 || sj >= g.ny) return 2 * yz + (wj == 0 ? 0 : xz) + wi + (long long)g.nx * wk;
  return 2 * (yz + xz) + (wk == 0 ? 0 : xy) + wi + (long long)g.nx * wj;
}

template <class S>
__global__ void k_faith_snapshot(Pops<const S> a, Geo g, S* out) {
  const long long yz = (long long)g.ny * g.nz, xz = (long long)g.nx * g.nz, xy = (long long)g.nx * g.ny;
  const long long per = 2 * (yz + xz + xy), n = (long long)Q * per;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(e / per);
    long long r = e % per;
    int i, j, k;
    if (r < 2 * yz) {
      i = r < yz ? 0 : g.nx - 1;
      r %= yz;
      j = (int)(r % g.ny);
      k = (int)(r / g.ny);
    } else if (r < 2 * (yz + xz)) {
      r -= 2 * yz;
      j = r < xz ? 0 : g.ny - 1;
      r %= xz;
      i = (int)(r % g.nx);
      k = (int)(r / g.nx);
    } else {
      r -= 2 * (yz + xz);
      k = r < xy ? 0 : g.nz - 1;
      r %= xy;
      i = (int)(r % g.nx);
      j = (int)(r / g.nx);
    }
    out[e] = a.p[q][i + (long long)g.sx * (j + (long long)g.ny * k)];
  }
}

template <class F, int LAY, bool FAITH = false>
__global__ void __launch_bounds__(DIAG_THREADS) k_diag(Pops<const typename F::S> a, Geo g, double svisc,
                                                       double omega, typename F::R inv, double* partials,
                                                       typename F::R* vel, Halo<typename F::S> h,
                                                       const typename F::S* __restrict__ faith, int faith_zero) {
  using R = typename F::R; using V = typename F::V; using N = Num<V>;
  __shared__ KS sh[DIAG_THREADS];
  KS acc[ND];
#pragma unroll
  for (int d = 0; d < ND; ++d) acc[d] = {0.0, 0.0};
  const long long n = (long long)g.nx * g.ny * g.nz;
  const V svr = N::wrap((R)svisc);
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long long)g.nx * g.ny));
    V x[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
      x[q] = N::wrap(F::dec(a.p[ref_slot<LAY>(q)][ref_off<LAY>(g, q, i, j, k, 0, 0, 0)], inv));
    V ux, uy, uz;
    const V rho = moments<V>(x, ux, uy, uz);
    const V ke = N::c(0.5) * (ux * ux + uy * uy + uz * uz);
    kadd(acc[0], (double)N::raw(rho));
    kadd(acc[1], (double)N::raw(ux));
    kadd(acc[2], (double)N::raw(uy));
    kadd(acc[3], (double)N::raw(uz));
    kadd(acc[4], (double)N::raw(ke));
    if (!isfinite(N::raw(rho)) || !isfinite(N::raw(ux)) || !isfinite(N::raw(uy)) || !isfinite(N::raw(uz)))
      acc[8].s = __dadd_rn(acc[8].s, 1.0);
    if (vel) { vel[c] = N::raw(ux); vel[n + c] = N::raw(uy); vel[2 * n + c] = N::raw(uz); }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      // a z-slab pulls across its faces from its ghost planes
      const bool lo = czq(q) > 0 && k == 0, hi = czq(q) < 0 && k == g.nz - 1;
      const int si = i - cxq(q), sj = j - cyq(q), sk = k - czq(q);
      if (LAY == LAY_TWO && h.in_lo[0] && (lo || hi)) {
        const int po = wrapi(i - cxq(q), g.nx) + g.sx * wrapi(j - cyq(q), g.ny);
        x[q] = N::wrap(F::dec(lo ? h.in_lo[zslot(q)][po] : h.in_hi[zslot(q)][po], inv));
      } else if (FAITH && LAY == LAY_TWO &&
                 (si < 0 || si >= g.nx || sj < 0 || sj >= g.ny || sk < 0 || sk >= g.nz)) {
        // faithful mode: the reference's ghost cell of this pull, filled two
        // steps earlier (or never)
        const long long per = 2 * ((long long)g.ny * g.nz + (long long)g.nx * g.nz + (long long)g.nx * g.ny);
        x[q] = faith_zero ? N::c(0.0) : N::wrap(F::dec(faith[q * per + faith_off(g, si, sj, sk)], inv));
      } else {
        x[q] = N::wrap(F::dec(a.p[ref_slot<LAY>(q)][ref_off<LAY>(g, q, i, j, k, -cxq(q), -cyq(q), -czq(q))], inv));
      }
    }
    V e[Q], vx, vy, vz;
    const V rp = equilibrium<V>(x, e, vx, vy, vz);
    const V vsq = vx * vx + vy * vy + vz * vz;
    const V P = ptotal<V>(x, e);
    kadd(acc[5], (double)N::raw(N::c(0.5) * vsq));
    kadd(acc[6], (double)N::raw(N::c(2.0) * svr * P));
    const double r = (double)N::raw(rp);
    const double eps = __dmul_rn(__dmul_rn(__dmul_rn(2.0, svisc), __ddiv_rn(__dmul_rn(__dmul_rn(9.0, omega), omega),
                                                                          __dmul_rn(__dmul_rn(4.0, r), r))),
                                 (double)N::raw(P));
    kadd(acc[7], eps);
  }
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    const KS r = block_reduce(acc[d], sh);
    if (threadIdx.x == 0) {
      partials[(blockIdx.x * ND + d) * 2 + 0] = r.s;
      partials[(blockIdx.x * ND + d) * 2 + 1] = r.c;
    }
  }
}

template <class R>
__global__ void __launch_bounds__(DIAG_THREADS) k_enstrophy(const R* __restrict__ vel, int nx, int ny, int nz,
                                                            double* partials) {
  __shared__ KS sh[DIAG_THREADS];
  KS acc = {0.0, 0.0};
  const long long n = (long long)nx * ny * nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
    const int ip = i + 1 == nx ? 0 : i + 1, im = i == 0 ? nx - 1 : i - 1;
    const int jp = j + 1 == ny ? 0 : j + 1, jm = j == 0 ? ny - 1 : j - 1;
    const int kp = k + 1 == nz ? 0 : k + 1, km = k == 0 ? nz - 1 : k - 1;
    auto U = [&](int comp, int a, int b, int d) -> double {
      return (double)vel[comp * n + a + (long long)nx * (b + (long long)ny * d)];
    };
    using E = Ex<double>;
    const E h = {0.5};
    const E dwdy = h * (E{U(2, i, jp, k)} - E{U(2, i, jm, k)});
    const E dvdz = h * (E{U(1, i, j, kp)} - E{U(1, i, j, km)});
    const E dudz = h * (E{U(0, i, j, kp)} - E{U(0, i, j, km)});
    const E dwdx = h * (E{U(2, ip, j, k)} - E{U(2, im, j, k)});
    const E dvdx = h * (E{U(1, ip, j, k)} - E{U(1, im, j, k)});
    const E dudy = h * (E{U(0, i, jp, k)} - E{U(0, i, jm, k)});
    const E wx = dwdy - dvdz, wy = dudz - dwdx, wz = dvdx - dudy;
    kadd(acc, (h * (wx * wx + wy * wy + wz * wz)).v);
  }
  const KS r = block_reduce(acc, sh);
  if (threadIdx.x == 0) {
    partials[(blockIdx.x * ND + 9) * 2 + 0] = r.s;
    partials[(blockIdx.x * ND + 9) * 2 + 1] = r.c;
  }
}

__global__ void __launch_bounds__(DIAG_THREADS) k_finalize(const double* __restrict__ partials, double* totals) {
  __shared__ KS sh[DIAG_THREADS];
  for (int d = 0; d < ND; ++d) {
    KS acc = {0.0, 0.0};
    for (int b = threadIdx.x; b < DIAG_BLOCKS; b += blockDim.x)
      kcomb(acc, KS{partials[(b * ND + d) * 2], partials[(b * ND + d) * 2 + 1]});
    const KS r = block_reduce(acc, sh);
    if (threadIdx.x == 0) totals[d] = __dadd_rn(r.s, r.c);
  }
}

template <class F, int LAY>
__global__ void k_last_zj(Pops<const typename F::S> a, Geo g, typename F::R inv, double* out) {
  using V = typename F::V; using N = Num<V>;
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  V x[Q];
  for (int q = 0; q < Q; ++q)
    x[q] = N::wrap(F::dec(a.p[ref_slot<LAY>(q)][ref_off<LAY>(g, q, g.nx - 1, g.ny - 1, g.nz - 1, 0, 0, 0)], inv));
  V ux, uy, uz;
  (void)moments<V>(x, ux, uy, uz);
  *out = (double)N::raw(uz);
}

// -------------------------------------------------------------------- VTK
// Velocity j/rho of the points of a VTK slice or box, as float triples in the
// file order of SRC/vtk_xy.binary.F90:79-97 (xy: j outer, i inner), vtk_xz
// (k, i), vtk_yz (k, j) and vtk_3d (k, j, i). The sums are taken in the
// storage arithmetic in the reference's order, each rounded to single
// precision, then divided in single precision (u/den).
template <class F, int LAY>
__global__ void k_vtk(Pops<const typename F::S> a, Geo g, int kind, int index, float* out, long long npts,
                      typename F::R inv) {
  using V = typename F::V; using N = Num<V>;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < npts; c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    if (kind == 1) { i = (int)(c % g.nx); j = (int)(c / g.nx); k = index; }
    else if (kind == 2) { i = (int)(c % g.nx); k = (int)(c / g.nx); j = index; }
    else if (kind == 3) { j = (int)(c % g.ny); k = (int)(c / g.ny); i = index; }
    else { i = (int)(c % g.nx); j = (int)((c / g.nx) % g.ny); k = (int)(c / ((long long)g.nx * g.ny)); }
    V x[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) x[q] = N::wrap(F::dec(a.p[ref_slot<LAY>(q)][ref_off<LAY>(g, q, i, j, k, 0, 0, 0)], inv));
    const V u = x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13];
    const V w = x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17];
    const V v = x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15];
    const V den = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7] + x[8] + x[9] + x[10] + x[11] + x[12] +
                  x[13] + x[14] + x[15] + x[16] + x[17] + x[18] + N::c(1.0);
    const float d = (float)N::raw(den);
    out[3 * c + 0] = __fdiv_rn((float)N::raw(u), d);
    out[3 * c + 1] = __fdiv_rn((float)N::raw(w), d);
    out[3 * c + 2] = __fdiv_rn((float)N::raw(v), d);
  }
}

// --------------------------------------------------------------- spectrum
template <class C>
__global__ void k_spec_bins(const C* __restrict__ f, int nx, int ny, int nz, int nbins, double* bins, double norm) {
  const int nxh = nx / 2 + 1;
  const long long n = (long long)nxh * ny * nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(c % nxh), iy = (int)((c / nxh) % ny), iz = (int)(c / ((long long)nxh * ny));
    const int ky = iy <= ny / 2 ? iy : iy - ny, kz = iz <= nz / 2 ? iz : iz - nz;
    // modes 0 < kx < nx/2 stand for their conjugate partner as well
    const double w = (ix == 0 || (nx % 2 == 0 && ix == nx / 2)) ? 1.0 : 2.0;
    const double kk = sqrt((double)ix * ix + (double)ky * ky + (double)kz * kz);
    const int b = (int)floor(kk + 0.5);
    if (b < nbins) {
      const double re = (double)f[c].x, im = (double)f[c].y;
      atomicAdd(bins + b, w * 0.5 * (re * re + im * im) * norm);
    }
  }
}

cudaError_t launch_spectrum_bins(const void* fft_out, int form, int nx, int ny, int nz, int nbins, double* bins,
                                 double norm, cudaStream_t st) {
  const long long n = (long long)(nx / 2 + 1) * ny * nz;
  const int grid = grid_1d(n, 256, 148 * 16);
  if (form == FORM_F64)
    k_spec_bins<double2><<<grid, 256, 0, st>>>((const double2*)fft_out, nx, ny, nz, nbins, bins, norm);
  else
    k_spec_bins<float2><<<grid, 256, 0, st>>>((const float2*)fft_out, nx, ny, nz, nbins, bins, norm);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- shift3
template <class T>
__global__ void k_shift3(const T* __restrict__ i1, const T* __restrict__ i2, const T* __restrict__ i3, T* o1, T* o2,
                         T* o3, int nx, int ny, int nz, int dir) {
  const long long n = (long long)nx * ny * nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
    const long long rowj = (long long)nx * (j + (long long)ny * k);
    const int is = wrapi(i - dir, nx), js = wrapi(j - dir, ny), ks = wrapi(k - dir, nz);
    o1[c] = __ldg(i1 + rowj + is);
    o2[c] = __ldg(i2 + i + (long long)nx * (js + (long long)ny * k));
    o3[c] = __ldg(i3 + i + (long long)nx * (j + (long long)ny * ks));
  }
}

// ============================================================== launchers
template <class S> static Pops<S> pops_of(const Lattice& L) {
  Pops<S> p;
  for (int q = 0; q < Q; ++q) p.p[q] = (S*)L.p[q];
  return p;
}

StepK make_stepk(int form, double omega, double scale, double les_cs) {
  StepK k{};
  k.omega = omega;
  k.omega_f = (float)omega;
  k.inv = (float)(1.0 / scale);
  k.om1 = 1.0f - (float)omega;
  k.scale = (float)scale;
  const double w[3] = {1.0 / 3.0, 1.0 / 18.0, 1.0 / 36.0};
  for (int c = 0; c < 3; ++c) k.kw[c] = (float)((double)(float)omega * scale * w[c]);
  // Smagorinsky constants of SRC/col_MC.F90:305 in the form's arithmetic:
  // 18*(cteS)**2, 1/(2*omega1) and (1/omega1)**2 (host code is built without
  // contraction, so each operation rounds as written)
  k.les = les_cs > 0.0;
  if (k.les) {
    k.cs18 = 18.0 * (les_cs * les_cs);
    k.tauh = 1.0 / (2.0 * omega);
    k.tau2 = (1.0 / omega) * (1.0 / omega);
    const float cs = (float)les_cs, om = (float)omega;
    k.cs18_f = 18.0f * (cs * cs);
    k.tauh_f = 1.0f / (2.0f * om);
    k.tau2_f = (1.0f / om) * (1.0f / om);
  }
  (void)form;
  return k;
}

// Grid of the several-cells-per-thread kernels: 128-thread blocks over the
// ny * 2^log_tpr threads of a plane, `planes` planes.
static dim3 vec_grid(const Geo& g, int log_tpr, int planes) {
  return dim3((unsigned)((((long long)g.ny << log_tpr) + 127) / 128), (unsigned)planes);
}

// log2(nx/V) when a V-cells-per-thread kernel applies (nx/V a power of two,
// whole warps per plane), else -1.
static int vec_log_tpr(const Geo& g, int V) {
  if (g.nx % V) return -1;
  const int tpr = g.nx / V;
  if (tpr & (tpr - 1)) return -1;
  if (((long long)g.ny * tpr) % 32) return -1;
  int l = 0;
  while ((1 << l) < tpr) ++l;
  return l;
}

template <class F>
static cudaError_t two_impl(const Lattice& s, const Lattice& d, const StepK& K, int variant, cudaStream_t st) {
  using S = typename F::S;
  Pops<const S> ps = pops_of<const S>(s);
  Pops<S> pd = pops_of<S>(d);
  pd.p[Q - 1] = (S*)s.p[Q - 1];  // pop 19 in place (SRC/col_MC.F90:351)
  Shape sh = cell_shape(s.g);
  // FP32: two cells per thread where the box fits it (automatic or 2): on
  // B200 at 256^3, 43.7 GLUPS against 42.0 with one cell per thread, the
  // Smagorinsky step 43.5 against 40.7
  const int lt2 = F::id == FORM_F32 && (variant == 0 || variant == 2) ? vec_log_tpr(s.g, 2) : -1;
  if (lt2 >= 0) {
    Pops<float> pf = pops_of<float>(d);
    pf.p[Q - 1] = (float*)s.p[Q - 1];
    const dim3 grid = vec_grid(s.g, lt2, s.g.nz);
    if (K.les) k_two_f32v<true><<<grid, 128, 0, st>>>(pops_of<const float>(s), pf, s.g, K, lt2, 0);
    else k_two_f32v<false><<<grid, 128, 0, st>>>(pops_of<const float>(s), pf, s.g, K, lt2, 0);
    return cudaGetLastError();
  }
  if (K.les) {  // the Smagorinsky collision: one cell per thread, FP16 four where the box fits
    const int lt = F::id == FORM_F16 && (variant == 0 || variant == 4) ? vec_log_tpr(s.g, 4) : -1;
    if (lt >= 0) {
      Pops<__half> ph = pops_of<__half>(d);
      ph.p[Q - 1] = (__half*)s.p[Q - 1];
      const dim3 grid = vec_grid(s.g, lt, s.g.nz);
      k_two_f16v<true><<<grid, 128, 0, st>>>(pops_of<const __half>(s), ph, s.g, K, lt, 0);
    } else {
      k_two<F, true><<<sh.grid, sh.block, 0, st>>>(ps, pd, s.g, K);
    }
    return cudaGetLastError();
  }
  if (variant == 8) {
    bool launched = false;
    cudaError_t e = launch_rows(s, d, ROW_TWO, K, st, &launched);
    if (e != cudaSuccess || launched) return e;
  }
  // automatic choice (variant 0): one cell per thread for FP64, two for FP32
  // (above), four cells per thread for FP16 where the box fits it - the fastest measured on
  // B200 at 256^3 (FP16: 76.6 GLUPS with four cells per thread against 64.0
  // with one, 62.7 with two and 44.6 for the row pipeline)
  if (F::id == FORM_F16 && (variant == 2 || variant == 4 || variant == 0)) {
    const int V = variant == 0 ? 4 : variant;
    const int lt = vec_log_tpr(s.g, V);
    if (lt >= 0) {
      const long long threads = (long long)s.g.ny << lt;
      dim3 grid((unsigned)((threads + (V == 4 ? 127 : 255)) / (V == 4 ? 128 : 256)), s.g.nz);
      Pops<__half> ph = pops_of<__half>(d);
      ph.p[Q - 1] = (__half*)s.p[Q - 1];
      if (V == 4) k_two_f16v<false><<<grid, 128, 0, st>>>(pops_of<const __half>(s), ph, s.g, K, lt, 0);
      else k_two_f16v2<<<grid, 256, 0, st>>>(pops_of<const __half>(s), ph, s.g, K, lt);
      return cudaGetLastError();
    }
  }
  k_two<F><<<sh.grid, sh.block, 0, st>>>(ps, pd, s.g, K);
  return cudaGetLastError();
}

cudaError_t launch_step_out_of_place(const Lattice& src, const Lattice& dst, double omega, cudaStream_t st) {
  const StepK K = make_stepk(src.form, omega, 1.0);
  const Shape sh = cell_shape(src.g);
  switch (src.form) {
    case FORM_F64:
      k_two<F64><<<sh.grid, sh.block, 0, st>>>(pops_of<const double>(src), pops_of<double>(dst), src.g, K);
      return cudaGetLastError();
    case FORM_F32: {
      const int lt2 = vec_log_tpr(src.g, 2);
      if (lt2 >= 0)
        k_two_f32v<false><<<vec_grid(src.g, lt2, src.g.nz), 128, 0, st>>>(pops_of<const float>(src),
                                                                           pops_of<float>(dst), src.g, K, lt2, 0);
      else
        k_two<F32><<<sh.grid, sh.block, 0, st>>>(pops_of<const float>(src), pops_of<float>(dst), src.g, K);
      return cudaGetLastError();
    }
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_two_lattice(const Lattice& src, const Lattice& dst, double omega, double scale, double les_cs,
                               int variant, cudaStream_t st) {
  const StepK K = make_stepk(src.form, omega, scale, les_cs);
  switch (src.form) {
    case FORM_F64: return two_impl<F64>(src, dst, K, variant, st);
    case FORM_F32: return two_impl<F32>(src, dst, K, variant, st);
    case FORM_F16: return two_impl<F16>(src, dst, K, variant, st);
  }
  return cudaErrorInvalidValue;
}

template <class F>
static cudaError_t aa_impl(const Lattice& a, int odd, const StepK& K, int variant, cudaStream_t st) {
  using S = typename F::S;
  Shape sh = cell_shape(a.g);
  const int lt4 = F::id == FORM_F16 && (variant == 0 || variant == 4) ? vec_log_tpr(a.g, 4) : -1;
  // FP32: two cells per thread where the box fits it (automatic or 2): on
  // B200 the pair of AA steps measured 41.9 GLUPS against 39.8 with one cell
  // per thread at 256^3 (40.5 against 38.9 at 1024^3), the Smagorinsky pair
  // 40.6 against 34.1
  const int lt2 = F::id == FORM_F32 && (variant == 0 || variant == 2) ? vec_log_tpr(a.g, 2) : -1;
  // FP32 odd step (automatic): four cells per thread where the box fits it;
  // the pair of AA steps measured 44.1 GLUPS at 256^3 and 44.2 at 512^3
  // against 42.2 and 40.8 with two cells per thread on both steps, and with
  // the Smagorinsky collision 43.9 against 40.9 at 256^3 (in FP16 eight cells
  // gave the Smagorinsky odd step nothing: 76.0 against 76.2, issue-bound)
  const int lt4f = F::id == FORM_F32 && variant == 0 && odd ? vec_log_tpr(a.g, 4) : -1;
  if (lt4f >= 0) {
    const dim3 grid = vec_grid(a.g, lt4f, a.g.nz);
    if (K.les) k_aa_f32w<true><<<grid, 128, 0, st>>>(pops_of<float>(a), a.g, K, lt4f);
    else k_aa_f32w<false><<<grid, 128, 0, st>>>(pops_of<float>(a), a.g, K, lt4f);
    return cudaGetLastError();
  }
  if (lt2 >= 0) {
    const dim3 grid = vec_grid(a.g, lt2, a.g.nz);
    Pops<float> pf = pops_of<float>(a);
    if (K.les) {
      if (odd) k_aa_f32v<true, true><<<grid, 128, 0, st>>>(pf, a.g, K, lt2);
      else k_aa_f32v<false, true><<<grid, 128, 0, st>>>(pf, a.g, K, lt2);
    } else {
      if (odd) k_aa_f32v<true, false><<<grid, 128, 0, st>>>(pf, a.g, K, lt2);
      else k_aa_f32v<false, false><<<grid, 128, 0, st>>>(pf, a.g, K, lt2);
    }
    return cudaGetLastError();
  }
  if (K.les) {
    if (lt4 >= 0) {
      const dim3 grid = vec_grid(a.g, lt4, a.g.nz);
      if (odd) k_aa_f16v<true, true><<<grid, 128, 0, st>>>(pops_of<__half>(a), a.g, K, lt4);
      else k_aa_f16v<false, true><<<grid, 128, 0, st>>>(pops_of<__half>(a), a.g, K, lt4);
    } else if (odd) {
      k_aa<F, true, true><<<sh.grid, sh.block, 0, st>>>(pops_of<S>(a), a.g, K);
    } else {
      k_aa<F, false, true><<<sh.grid, sh.block, 0, st>>>(pops_of<S>(a), a.g, K);
    }
    return cudaGetLastError();
  }
  if (variant == 8) {
    bool launched = false;
    cudaError_t e = launch_rows(a, a, odd ? ROW_AA_ODD : ROW_AA_EVEN, K, st, &launched);
    if (e != cudaSuccess || launched) return e;
  }
  // FP16 odd step (automatic): eight cells per thread where the box fits it.
  // On B200 the pair of AA steps measured 84.3 GLUPS at 256^3 and 86.0 at
  // 512^3 against 80.0 and 81.6 with four cells per thread on both steps;
  // eight cells on the even step as well measured the same (84.1, 86.1), so
  // the even step stays on k_aa_f16v (96 registers, 5 blocks/SM)
  const int lt8 = F::id == FORM_F16 && variant == 0 && odd ? vec_log_tpr(a.g, 8) : -1;
  if (lt8 >= 0) {
    k_aa_f16w<true><<<vec_grid(a.g, lt8, a.g.nz), 128, 0, st>>>(pops_of<__half>(a), a.g, K, lt8);
    return cudaGetLastError();
  }
  // FP16: four cells per thread where the box fits it (automatic or 4)
  if (lt4 >= 0) {
    const dim3 grid = vec_grid(a.g, lt4, a.g.nz);
    if (odd) k_aa_f16v<true, false><<<grid, 128, 0, st>>>(pops_of<__half>(a), a.g, K, lt4);
    else k_aa_f16v<false, false><<<grid, 128, 0, st>>>(pops_of<__half>(a), a.g, K, lt4);
    return cudaGetLastError();
  }
  if (odd && F::id == FORM_F16)
    k_aa_f16_odd<<<sh.grid, sh.block, 0, st>>>(pops_of<__half>(a), a.g, K);
  else if (odd) k_aa<F, true><<<sh.grid, sh.block, 0, st>>>(pops_of<S>(a), a.g, K);
  else k_aa<F, false><<<sh.grid, sh.block, 0, st>>>(pops_of<S>(a), a.g, K);
  return cudaGetLastError();
}

cudaError_t launch_aa(const Lattice& a, int odd, double omega, double scale, double les_cs, int variant,
                      cudaStream_t st) {
  const StepK K = make_stepk(a.form, omega, scale, les_cs);
  switch (a.form) {
    case FORM_F64: return aa_impl<F64>(a, odd, K, variant, st);
    case FORM_F32: return aa_impl<F32>(a, odd, K, variant, st);
    case FORM_F16: return aa_impl<F16>(a, odd, K, variant, st);
  }
  return cudaErrorInvalidValue;
}

template <class F>
static cudaError_t tgv_impl(const Lattice& a, int lay, double u0, int faithful, double scale, unsigned int* mx,
                            cudaStream_t st) {
  using S = typename F::S; using R = typename F::R;
  const long long n = (long long)a.g.nx * a.g.ny * a.g.nz;
  k_init_tgv<F><<<grid_1d(n, 256, 148 * 32), 256, 0, st>>>(pops_of<S>(a), a.g, lay, (R)u0, faithful, (R)scale, mx);
  return cudaGetLastError();
}

cudaError_t launch_init_tgv(const Lattice& a, int lay, double u0, int faithful, double scale, unsigned int* mx,
                            cudaStream_t st) {
  switch (a.form) {
    case FORM_F64: return tgv_impl<F64>(a, lay, u0, faithful, scale, mx, st);
    case FORM_F32: return tgv_impl<F32>(a, lay, u0, faithful, scale, mx, st);
    case FORM_F16: return tgv_impl<F16>(a, lay, u0, faithful, scale, mx, st);
  }
  return cudaErrorInvalidValue;
}

template <class F>
static cudaError_t vel_impl(const Lattice& a, int lay, const double* u, const double* v, const double* w, double rho,
                            int k0, int nk, double scale, unsigned int* mx, cudaStream_t st) {
  using S = typename F::S; using R = typename F::R;
  const long long n = (long long)a.g.nx * a.g.ny * nk;
  k_init_vel<F><<<grid_1d(n, 256, 148 * 32), 256, 0, st>>>(pops_of<S>(a), a.g, lay, u, v, w, rho, k0, nk, (R)scale,
                                                           mx);
  return cudaGetLastError();
}

cudaError_t launch_init_velocity(const Lattice& a, int lay, const double* u, const double* v, const double* w,
                                 double rho, int k0, int nk, double scale, unsigned int* mx, cudaStream_t st) {
  switch (a.form) {
    case FORM_F64: return vel_impl<F64>(a, lay, u, v, w, rho, k0, nk, scale, mx, st);
    case FORM_F32: return vel_impl<F32>(a, lay, u, v, w, rho, k0, nk, scale, mx, st);
    case FORM_F16: return vel_impl<F16>(a, lay, u, v, w, rho, k0, nk, scale, mx, st);
  }
  return cudaErrorInvalidValue;
}

template <class F, int LAY>
static void export_lay(const Lattice& a, int q, void* ds, double* dd, double scale, cudaStream_t st) {
  using S = typename F::S; using R = typename F::R;
  const long long n = (long long)a.g.nx * a.g.ny * a.g.nz;
  k_export<F, LAY><<<grid_1d(n, 256, 148 * 32), 256, 0, st>>>(pops_of<const S>(a), a.g, q, (S*)ds, dd,
                                                               (R)(1.0 / scale));
}
template <class F>
static cudaError_t export_impl(const Lattice& a, int lay, int q, void* ds, double* dd, double scale, cudaStream_t st) {
  if (lay == LAY_TWO) export_lay<F, LAY_TWO>(a, q, ds, dd, scale, st);
  else if (lay == LAY_AAE) export_lay<F, LAY_AAE>(a, q, ds, dd, scale, st);
  else export_lay<F, LAY_AAN>(a, q, ds, dd, scale, st);
  return cudaGetLastError();
}
cudaError_t launch_export(const Lattice& a, int lay, int q, void* ds, double* dd, double scale, cudaStream_t st) {
  switch (a.form) {
    case FORM_F64: return export_impl<F64>(a, lay, q, ds, dd, scale, st);
    case FORM_F32: return export_impl<F32>(a, lay, q, ds, dd, scale, st);
    case FORM_F16: return export_impl<F16>(a, lay, q, ds, dd, scale, st);
  }
  return cudaErrorInvalidValue;
}

template <class F, int LAY>
static void import_lay(const Lattice& a, int q, const void* ds, cudaStream_t st) {
  using S = typename F::S;
  const long long n = (long long)a.g.nx * a.g.ny * a.g.nz;
  k_import<F, LAY><<<grid_1d(n, 256, 148 * 32), 256, 0, st>>>(pops_of<S>(a), a.g, q, (const S*)ds);
}
template <class F>
static cudaError_t import_impl(const Lattice& a, int lay, int q, const void* ds, cudaStream_t st) {
  if (lay == LAY_TWO) import_lay<F, LAY_TWO>(a, q, ds, st);
  else if (lay == LAY_AAE) import_lay<F, LAY_AAE>(a, q, ds, st);
  else import_lay<F, LAY_AAN>(a, q, ds, st);
  return cudaGetLastError();
}
cudaError_t launch_import(const Lattice& a, int lay, int q, const void* ds, cudaStream_t st) {
  switch (a.form) {
    case FORM_F64: return import_impl<F64>(a, lay, q, ds, st);
    case FORM_F32: return import_impl<F32>(a, lay, q, ds, st);
    case FORM_F16: return import_impl<F16>(a, lay, q, ds, st);
  }
  return cudaErrorInvalidValue;
}

template <class S> static Halo<S> halo_of(const SlabLinks* l) {
  Halo<S> h{};
  if (!l) return h;
  for (int s = 0; s < NZF; ++s) {
    h.in_lo[s] = (const S*)l->in_lo[s];
    h.in_hi[s] = (const S*)l->in_hi[s];
    h.up[s] = (S*)l->up[s];
    h.dn[s] = (S*)l->dn[s];
  }
  return h;
}

template <class F, int LAY>
static void diag_lay(const Lattice& a, double svisc, double omega, double scale, double* partials, void* vel,
                     const SlabLinks* halo, const void* faith, bool fzero, cudaStream_t st) {
  using S = typename F::S; using R = typename F::R;
  if (faith || fzero)
    k_diag<F, LAY, true><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(pops_of<const S>(a), a.g, svisc, omega,
                                                             (R)(1.0 / scale), partials, (R*)vel, halo_of<S>(halo),
                                                             (const S*)faith, fzero ? 1 : 0);
  else
    k_diag<F, LAY><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(pops_of<const S>(a), a.g, svisc, omega, (R)(1.0 / scale),
                                                         partials, (R*)vel, halo_of<S>(halo), nullptr, 0);
}
template <class F>
static cudaError_t diag_impl(const Lattice& a, int lay, double svisc, double omega, double scale, double* partials,
                             void* vel, const SlabLinks* halo, const void* faith, bool fzero, cudaStream_t st) {
  if (lay == LAY_TWO) diag_lay<F, LAY_TWO>(a, svisc, omega, scale, partials, vel, halo, faith, fzero, st);
  else if (lay == LAY_AAE) diag_lay<F, LAY_AAE>(a, svisc, omega, scale, partials, vel, halo, nullptr, false, st);
  else diag_lay<F, LAY_AAN>(a, svisc, omega, scale, partials, vel, halo, nullptr, false, st);
  return cudaGetLastError();
}

long long faith_planes_elems(const Geo& g) {
  return (long long)Q * 2 * ((long long)g.ny * g.nz + (long long)g.nx * g.nz + (long long)g.nx * g.ny);
}

cudaError_t launch_faith_snapshot(const Lattice& a, void* out, cudaStream_t st) {
  const long long n = faith_planes_elems(a.g);
  const int blocks = grid_1d(n, 256, 148 * 16);
  switch (a.form) {
    case FORM_F64: k_faith_snapshot<double><<<blocks, 256, 0, st>>>(pops_of<const double>(a), a.g, (double*)out); break;
    case FORM_F32: k_faith_snapshot<float><<<blocks, 256, 0, st>>>(pops_of<const float>(a), a.g, (float*)out); break;
    case FORM_F16: k_faith_snapshot<__half><<<blocks, 256, 0, st>>>(pops_of<const __half>(a), a.g, (__half*)out); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}
cudaError_t launch_diag(const Lattice& a, int lay, double svisc, double omega, double scale, double* partials,
                        void* vel, cudaStream_t st, const SlabLinks* halo, const void* faith, bool faith_zero) {
  switch (a.form) {
    case FORM_F64: return diag_impl<F64>(a, lay, svisc, omega, scale, partials, vel, halo, faith, faith_zero, st);
    case FORM_F32: return diag_impl<F32>(a, lay, svisc, omega, scale, partials, vel, halo, faith, faith_zero, st);
    case FORM_F16: return diag_impl<F16>(a, lay, svisc, omega, scale, partials, vel, halo, faith, faith_zero, st);
  }
  return cudaErrorInvalidValue;
}

template <class F>
static cudaError_t slab_impl(const Lattice& s, const Lattice& d, const StepK& K, const SlabLinks& l,
                             cudaStream_t st, cudaStream_t st_in) {
  using S = typename F::S;
  Pops<const S> ps = pops_of<const S>(s);
  Pops<S> pd = pops_of<S>(d);
  pd.p[Q - 1] = (S*)s.p[Q - 1];  // pop 19 in place (SRC/col_MC.F90:351)
  const Shape sh = cell_shape(s.g);
  const Halo<S> h = halo_of<S>(&l);
  // planes 0 and nz-1 (one plane when nz = 1) on st, the interior on st_in:
  // the two read only the source lattice and write disjoint planes, so they
  // may run side by side
  const dim3 ge(sh.grid.x, sh.grid.y, s.g.nz > 1 ? 2 : 1);
  if (K.les) k_slab<F, true, true><<<ge, sh.block, 0, st>>>(ps, pd, s.g, K, h);
  else k_slab<F, false, true><<<ge, sh.block, 0, st>>>(ps, pd, s.g, K, h);
  if (s.g.nz > 2) {
    // FP16 / FP32: the interior planes on the four- / two-cells-per-thread
    // kernel where the rows fit it (planes 1 .. nz-2 pull only inside the
    // slab, so its z wrap never applies)
    const int lt = F::id == FORM_F16 ? vec_log_tpr(s.g, 4) : -1;
    const int lt2 = F::id == FORM_F32 ? vec_log_tpr(s.g, 2) : -1;
    if (lt2 >= 0) {
      Pops<float> pf = pops_of<float>(d);
      pf.p[Q - 1] = (float*)s.p[Q - 1];
      const dim3 gv = vec_grid(s.g, lt2, s.g.nz - 2);
      if (K.les) k_two_f32v<true><<<gv, 128, 0, st_in>>>(pops_of<const float>(s), pf, s.g, K, lt2, 1);
      else k_two_f32v<false><<<gv, 128, 0, st_in>>>(pops_of<const float>(s), pf, s.g, K, lt2, 1);
    } else if (lt >= 0) {
      Pops<__half> ph = pops_of<__half>(d);
      ph.p[Q - 1] = (__half*)s.p[Q - 1];
      const dim3 gv = vec_grid(s.g, lt, s.g.nz - 2);
      if (K.les) k_two_f16v<true><<<gv, 128, 0, st_in>>>(pops_of<const __half>(s), ph, s.g, K, lt, 1);
      else k_two_f16v<false><<<gv, 128, 0, st_in>>>(pops_of<const __half>(s), ph, s.g, K, lt, 1);
    } else {
      const dim3 gi(sh.grid.x, sh.grid.y, s.g.nz - 2);
      if (K.les) k_slab<F, true, false><<<gi, sh.block, 0, st_in>>>(ps, pd, s.g, K, h);
      else k_slab<F, false, false><<<gi, sh.block, 0, st_in>>>(ps, pd, s.g, K, h);
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_slab(const Lattice& src, const Lattice& dst, const SlabLinks& links, double omega, double scale,
                        double les_cs, cudaStream_t st, cudaStream_t st_interior) {
  const StepK K = make_stepk(src.form, omega, scale, les_cs);
  switch (src.form) {
    case FORM_F64: return slab_impl<F64>(src, dst, K, links, st, st_interior);
    case FORM_F32: return slab_impl<F32>(src, dst, K, links, st, st_interior);
    case FORM_F16: return slab_impl<F16>(src, dst, K, links, st, st_interior);
  }
  return cudaErrorInvalidValue;
}

template <class S>
static cudaError_t prime_impl(const Lattice& a, const SlabLinks& l, cudaStream_t st) {
  const int tx = a.g.nx >= 256 ? 256 : ((a.g.nx + 31) / 32) * 32;
  k_halo_prime<S><<<dim3((a.g.nx + tx - 1) / tx, a.g.ny), tx, 0, st>>>(pops_of<const S>(a), a.g, halo_of<S>(&l));
  return cudaGetLastError();
}

cudaError_t launch_halo_prime(const Lattice& a, const SlabLinks& links, cudaStream_t st) {
  switch (a.form) {
    case FORM_F64: return prime_impl<double>(a, links, st);
    case FORM_F32: return prime_impl<float>(a, links, st);
    case FORM_F16: return prime_impl<__half>(a, links, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_enstrophy(const Lattice& a, const void* vel, double* partials, cudaStream_t st) {
  if (a.form == FORM_F64)
    k_enstrophy<double><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>((const double*)vel, a.g.nx, a.g.ny, a.g.nz, partials);
  else
    k_enstrophy<float><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>((const float*)vel, a.g.nx, a.g.ny, a.g.nz, partials);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const double* partials, double* totals, cudaStream_t st) {
  k_finalize<<<1, DIAG_THREADS, 0, st>>>(partials, totals);
  return cudaGetLastError();
}

template <class F>
static cudaError_t lastzj_impl(const Lattice& a, int lay, double scale, double* out, cudaStream_t st) {
  using S = typename F::S; using R = typename F::R;
  const R inv = (R)(1.0 / scale);
  if (lay == LAY_TWO) k_last_zj<F, LAY_TWO><<<1, 32, 0, st>>>(pops_of<const S>(a), a.g, inv, out);
  else if (lay == LAY_AAE) k_last_zj<F, LAY_AAE><<<1, 32, 0, st>>>(pops_of<const S>(a), a.g, inv, out);
  else k_last_zj<F, LAY_AAN><<<1, 32, 0, st>>>(pops_of<const S>(a), a.g, inv, out);
  return cudaGetLastError();
}
cudaError_t launch_last_zj(const Lattice& a, int lay, double scale, double* out, cudaStream_t st) {
  switch (a.form) {
    case FORM_F64: return lastzj_impl<F64>(a, lay, scale, out, st);
    case FORM_F32: return lastzj_impl<F32>(a, lay, scale, out, st);
    case FORM_F16: return lastzj_impl<F16>(a, lay, scale, out, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_shift3(const void* const in[3], void* const out[3], int nx, int ny, int nz, int elem_bytes,
                          int reverse, cudaStream_t st) {
  const long long n = (long long)nx * ny * nz;
  const int grid = grid_1d(n, 256, 148 * 16);
  const int dir = reverse ? -1 : 1;
  if (elem_bytes == 8)
    k_shift3<double><<<grid, 256, 0, st>>>((const double*)in[0], (const double*)in[1], (const double*)in[2],
                                           (double*)out[0], (double*)out[1], (double*)out[2], nx, ny, nz, dir);
  else if (elem_bytes == 4)
    k_shift3<float><<<grid, 256, 0, st>>>((const float*)in[0], (const float*)in[1], (const float*)in[2],
                                          (float*)out[0], (float*)out[1], (float*)out[2], nx, ny, nz, dir);
  else if (elem_bytes == 2)
    k_shift3<__half><<<grid, 256, 0, st>>>((const __half*)in[0], (const __half*)in[1], (const __half*)in[2],
                                           (__half*)out[0], (__half*)out[1], (__half*)out[2], nx, ny, nz, dir);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

template <class F, int LAY>
static void vtk_lay(const Lattice& a, int kind, int index, float* out, long long npts, double scale,
                    cudaStream_t st) {
  using S = typename F::S; using R = typename F::R;
  k_vtk<F, LAY><<<grid_1d(npts, 256, 148 * 16), 256, 0, st>>>(pops_of<const S>(a), a.g, kind, index, out, npts,
                                                               (R)(1.0 / scale));
}
template <class F>
static cudaError_t vtk_impl(const Lattice& a, int lay, int kind, int index, float* out, long long npts, double scale,
                            cudaStream_t st) {
  if (lay == LAY_TWO) vtk_lay<F, LAY_TWO>(a, kind, index, out, npts, scale, st);
  else if (lay == LAY_AAE) vtk_lay<F, LAY_AAE>(a, kind, index, out, npts, scale, st);
  else vtk_lay<F, LAY_AAN>(a, kind, index, out, npts, scale, st);
  return cudaGetLastError();
}
cudaError_t launch_vtk(const Lattice& a, int lay, int kind, int index, float* out, long long npts, double scale,
                       cudaStream_t st) {
  switch (a.form) {
    case FORM_F64: return vtk_impl<F64>(a, lay, kind, index, out, npts, scale, st);
    case FORM_F32: return vtk_impl<F32>(a, lay, kind, index, out, npts, scale, st);
    case FORM_F16: return vtk_impl<F16>(a, lay, kind, index, out, npts, scale, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace bgk
