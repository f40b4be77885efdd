// Row-pipelined stream-collide: a persistent kernel that streams whole rows of
// all 19 populations into a ring of shared-memory stages with TMA bulk copies
// (cp.async.bulk global -> shared, completion on an mbarrier), several rows
// ahead of the computation, so that the bytes in flight do not depend on
// registers or occupancy.
//
// A task is a slab of R consecutive rows (j0..j0+R-1, k) of the box; CTAs take
// tasks round-robin. For each task and population the R source rows are
// copied whole (sx elements each, 16-byte aligned), in one bulk copy or two
// where the rows wrap around in j:
//   two-lattice: population q of the source lattice at row (j - cy, k - cz)
//                (SRC/col_MC.F90:113-131), pop 19 at (j, k);
//   AA even:     population q at row (j, k);
//   AA odd:      population opp(q) at row (j - cy, k - cz).
// The x-shift and the periodic wrap in x are resolved when a thread reads its
// cell from shared memory; results go straight to global memory. In the AA
// scheme every (population, row) pair is read and written by one task only,
// so prefetching rows of later tasks never races with the stores of earlier
// ones.
//
// Warp-specialised: one producer warp issues the copies into a ring of ns
// stages while the consumer warps compute; stages are handed over with
// mbarriers (full: copies landed; empty: all consumer warps done reading).
//
// Waits on an mbarrier are bounded: a wait that runs out sets *err; the
// producer then waits (bounded) for the copies it still has in flight and
// returns. With stall != 0 (test hook), the consumers of CTA 0 first wait on a
// barrier that nothing arms, so that this path can be exercised without a fault.
#include "kernels.h"

namespace bgk {

namespace {

constexpr int MAX_POLLS = 1 << 20;   // bound of a wait on row copies
constexpr int ROWS_MAX_THREADS = 32 + 512;  // producer warp + up to 16 consumer warps
constexpr int STALL_POLLS = 1 << 12; // bound of the injected wait (test hook)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int polls = MAX_POLLS) {
  for (int it = 0; it < polls; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ int wrapr(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Warp 0 is the producer (its lane 0 issues the bulk copies), warps 1..W the
// consumers. full[s] completes when the copies of stage s have landed;
// empty[s] completes when all W consumer warps have finished reading it.
template <class F, int MODE>
__global__ void __launch_bounds__(ROWS_MAX_THREADS) k_rows(Pops<typename F::S> src, Pops<typename F::S> dst, Geo g,
                                                           StepK K, int ns, int R, int* err, int stall) {
  using S = typename F::S;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned long long* full = reinterpret_cast<unsigned long long*>(smem);
  unsigned long long* empty = full + 8;
  unsigned long long* never = full + 15;  // never armed (test hook)
  S* stages = reinterpret_cast<S*>(smem + 128);
  const int sx = g.sx;
  const uint32_t rowbytes = (uint32_t)sx * (uint32_t)sizeof(S);
  const int slabs_y = g.ny / R;
  const int ntask = slabs_y * g.nz;
  const long long stage_elems = (long long)Q * R * sx;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nconsumer = (blockDim.x >> 5) - 1;
  if (threadIdx.x == 0) {
    for (int s = 0; s < ns; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), (uint32_t)nconsumer);
    }
    mbar_init(smem_u32(never), 1);
    mbar_fence_init();
  }
  __syncthreads();

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      int n = 0;
      bool bad = false;
      for (;; ++n) {
        const int t = blockIdx.x + n * gridDim.x;
        if (t >= ntask) break;
        const int s = n % ns;
        if (n >= ns && !mbar_wait(smem_u32(&empty[s]), (uint32_t)(((n / ns) - 1) & 1))) {
          bad = true;
          break;
        }
        const int j0 = (t % slabs_y) * R, k = t / slabs_y;
        const uint32_t bar = smem_u32(&full[s]);
        mbar_expect_tx(bar, (uint32_t)(Q * R) * rowbytes);
#pragma unroll 1
        for (int q = 0; q < Q; ++q) {
          int js = j0, kk = k, slot = q;
          if (MODE != ROW_AA_EVEN) {
            js = j0 - cyq(q);
            kk = wrapr(k - czq(q), g.nz);
          }
          if (MODE == ROW_AA_ODD) slot = oppq(q);
          const S* plane = src.p[slot] + (long long)sx * g.ny * kk;
          const uint32_t dst0 = smem_u32(stages + s * stage_elems + (long long)q * R * sx);
          // rows js .. js+R-1 of the plane, wrapped in j: at most two contiguous pieces
          if (js < 0) {
            bulk_g2s(dst0, plane + (long long)sx * (g.ny - 1), rowbytes, bar);
            if (R > 1) bulk_g2s(dst0 + rowbytes, plane, (uint32_t)(R - 1) * rowbytes, bar);
          } else if (js + R > g.ny) {
            if (R > 1) bulk_g2s(dst0, plane + (long long)sx * js, (uint32_t)(R - 1) * rowbytes, bar);
            bulk_g2s(dst0 + (uint32_t)(R - 1) * rowbytes, plane, rowbytes, bar);
          } else {
            bulk_g2s(dst0, plane + (long long)sx * js, (uint32_t)R * rowbytes, bar);
          }
        }
      }
      if (bad) {
        atomicExch(err, 1);
        // the copies of every stage filled since the consumers last released
        // it are still to land: wait (bounded) for them before returning
        for (int m = n - ns < 0 ? 0 : n - ns; m < n; ++m)
          (void)mbar_wait(smem_u32(&full[m % ns]), (uint32_t)((m / ns) & 1));
      }
    }
    return;
  }
  // -------------------------------------------------------------- consumers
  const int ctid = threadIdx.x - 32, nct = nconsumer * 32;
  const int cells = R * g.nx;
  for (int n = 0;; ++n) {
    const int t = blockIdx.x + n * gridDim.x;
    if (t >= ntask) break;
    const int s = n % ns;
    const bool stall_here = stall && blockIdx.x == 0 && n == 0;
    const bool ok = stall_here ? mbar_wait(smem_u32(never), 0u, STALL_POLLS)
                               : mbar_wait(smem_u32(&full[s]), (uint32_t)((n / ns) & 1));
    if (!ok) {
      if (lane == 0) atomicExch(err, 1);
      break;  // the producer's own bounded wait on empty[s] then ends it too
    }
    const int j0 = (t % slabs_y) * R, k = t / slabs_y;
    const S* st = stages + s * stage_elems;
    for (int c = ctid; c < cells; c += nct) {
      const int r = c / g.nx, i = c - r * g.nx;
      const int j = j0 + r;
      const int im = i == 0 ? g.nx - 1 : i - 1, ip = i == g.nx - 1 ? 0 : i + 1;
      S v[Q];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int ii = MODE == ROW_AA_EVEN ? i : (cxq(q) > 0 ? im : (cxq(q) < 0 ? ip : i));
        v[q] = st[(q * R + r) * sx + ii];
      }
      F::cell(v, K);
      if (MODE == ROW_TWO) {
        const long long o = i + (long long)sx * (j + (long long)g.ny * k);
#pragma unroll
        for (int q = 0; q < Q; ++q) dst.p[q][o] = v[q];
      } else if (MODE == ROW_AA_EVEN) {
        const long long o = i + (long long)sx * (j + (long long)g.ny * k);
#pragma unroll
        for (int q = 0; q < Q; ++q) dst.p[oppq(q)][o] = v[q];
      } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const int ii = cxq(q) > 0 ? ip : (cxq(q) < 0 ? im : i);
          const int jj = wrapr(j + cyq(q), g.ny), kk = wrapr(k + czq(q), g.nz);
          dst.p[q][ii + (long long)sx * (jj + (long long)g.ny * kk)] = v[q];
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_u32(&empty[s]));  // this warp is done with stage s
  }
}

template <class F, int MODE>
cudaError_t rows_impl(Pops<typename F::S> src, Pops<typename F::S> dst, const Geo& g, const StepK& K, int* err,
                      int stall, cudaStream_t st, bool* launched) {
  using S = typename F::S;
  *launched = false;
  // Slabs of R rows (R divides ny, at most 8) so that one bulk copy moves R
  // rows of a population; as many stages of about 100 KB in total as fit,
  // between 2 and 6.
  const size_t row = (size_t)g.sx * sizeof(S);
  int R = 1;
  while (R < 8 && g.ny % (2 * R) == 0 && (size_t)Q * 2 * R * row * 2 <= 100 * 1024) R *= 2;
  const size_t stage = (size_t)Q * R * row;
  int ns = (int)(100 * 1024 / stage);
  if (ns > 6) ns = 6;
  if (ns < 2) ns = 2;
  const size_t smem = 128 + (size_t)ns * stage;
  if (smem > 200 * 1024 || !err) return cudaSuccess;  // rows too long: caller uses another kernel
  const int threads = 32 + ((long long)R * g.nx > 256 ? 512 : 256);
  int dev = 0, nsm = 0, occ = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  static unsigned long long attr_set = 0;  // one bit per device ordinal
  if (dev < 64 && !((attr_set >> dev) & 1ULL)) {
    e = cudaFuncSetAttribute(k_rows<F, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    attr_set |= 1ULL << dev;
  }
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rows<F, MODE>, threads, smem);
  if (e != cudaSuccess) return e;
  if (occ < 1) return cudaSuccess;
  const int ntask = (g.ny / R) * g.nz;
  int grid = nsm * occ;
  if (grid > ntask) grid = ntask;
  k_rows<F, MODE><<<grid, threads, smem, st>>>(src, dst, g, K, ns, R, err, stall);
  *launched = true;
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_rows(const Lattice& src, const Lattice& dst, int mode, const StepK& K, cudaStream_t st,
                        bool* launched) {
  *launched = false;
  // every row must start on a 16-byte boundary and be a multiple of 16 bytes
  // long (sx is a multiple of 32 elements, population bases 256-element aligned)
  if (src.g.sx % 32) return cudaSuccess;
  switch (src.form) {
    case FORM_F64: {
      Pops<double> s, d;
      for (int q = 0; q < Q; ++q) { s.p[q] = (double*)src.p[q]; d.p[q] = (double*)dst.p[q]; }
      if (mode == ROW_TWO) { d.p[Q - 1] = s.p[Q - 1]; return rows_impl<F64, ROW_TWO>(s, d, src.g, K, src.err, src.stall, st, launched); }
      if (mode == ROW_AA_EVEN) return rows_impl<F64, ROW_AA_EVEN>(s, s, src.g, K, src.err, src.stall, st, launched);
      return rows_impl<F64, ROW_AA_ODD>(s, s, src.g, K, src.err, src.stall, st, launched);
    }
    case FORM_F32: {
      Pops<float> s, d;
      for (int q = 0; q < Q; ++q) { s.p[q] = (float*)src.p[q]; d.p[q] = (float*)dst.p[q]; }
      if (mode == ROW_TWO) { d.p[Q - 1] = s.p[Q - 1]; return rows_impl<F32, ROW_TWO>(s, d, src.g, K, src.err, src.stall, st, launched); }
      if (mode == ROW_AA_EVEN) return rows_impl<F32, ROW_AA_EVEN>(s, s, src.g, K, src.err, src.stall, st, launched);
      return rows_impl<F32, ROW_AA_ODD>(s, s, src.g, K, src.err, src.stall, st, launched);
    }
    case FORM_F16: {
      Pops<__half> s, d;
      for (int q = 0; q < Q; ++q) { s.p[q] = (__half*)src.p[q]; d.p[q] = (__half*)dst.p[q]; }
      if (mode == ROW_TWO) { d.p[Q - 1] = s.p[Q - 1]; return rows_impl<F16, ROW_TWO>(s, d, src.g, K, src.err, src.stall, st, launched); }
      if (mode == ROW_AA_EVEN) return rows_impl<F16, ROW_AA_EVEN>(s, s, src.g, K, src.err, src.stall, st, launched);
      return rows_impl<F16, ROW_AA_ODD>(s, s, src.g, K, src.err, src.stall, st, launched);
    }
  }
  return cudaErrorInvalidValue;
}

}  // namespace bgk
