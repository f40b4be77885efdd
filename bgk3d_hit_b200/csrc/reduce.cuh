// Deterministic compensated FP64 reductions shared by the diagnostics and
// the adjoint: Neumaier pairs per thread, fixed-order block trees.
#pragma once
#include <cuda_runtime.h>

namespace bgk {

struct KS { double s, c; };
// Neumaier step; explicit _rn operations keep it free of FMA contraction.
__device__ __forceinline__ void kadd(KS& a, double v) {
  const double t = __dadd_rn(a.s, v);
  if (fabs(a.s) >= fabs(v)) a.c = __dadd_rn(a.c, __dadd_rn(__dsub_rn(a.s, t), v));
  else a.c = __dadd_rn(a.c, __dadd_rn(__dsub_rn(v, t), a.s));
  a.s = t;
}
__device__ __forceinline__ void kcomb(KS& a, const KS& b) {
  kadd(a, b.s);
  a.c = __dadd_rn(a.c, b.c);
}

// Fixed-order block reduction of one quantity; thread 0 returns the result.
__device__ __forceinline__ KS block_reduce(KS v, KS* sh) {
  const int t = threadIdx.x;
  sh[t] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (t < s) { KS a = sh[t]; kcomb(a, sh[t + s]); sh[t] = a; }
    __syncthreads();
  }
  KS r = sh[0];
  __syncthreads();
  return r;
}

}  // namespace bgk
