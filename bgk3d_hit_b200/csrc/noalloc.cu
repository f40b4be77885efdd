// bgk_diagnostics_noalloc: the diagno + dissipation (+ strain-rate) reduction
// over caller-owned device populations, without allocating any memory.
//
// Why it exists: some callers of this library cannot call cudaMalloc once
// their time loop runs. A Fortran driver whose device arrays all live in an
// OpenACC data region owned by that runtime, or an application that hands all
// device memory to its own pool at start-up, must not have the library grab
// more: cudaMalloc can fail when the device is full and it synchronises the
// device. The context API (bgk_create) allocates its diagnostic buffers up
// front; this entry point needs no context and no allocation at all.
//
// Its only scratch is the file-scope device array below: the per-block
// compensated partial sums of the diagnostics reduction, a fixed
// NOALLOC_SCRATCH_BYTES (94,808 bytes) whatever the box size, because the
// reduction grid is fixed (DIAG_BLOCKS blocks of DIAG_THREADS threads, each
// thread striding over the cells). Every GPU that loads the library holds this
// array until the process exits.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>

#include "bgk3d.h"
#include "kernels.h"

using namespace bgk;

namespace {

// DIAG_BLOCKS x ND (sum, compensation) pairs, then ND + 1 totals.
constexpr size_t NOALLOC_PARTIALS = (size_t)DIAG_BLOCKS * ND * 2;
constexpr size_t NOALLOC_SCRATCH_DOUBLES = NOALLOC_PARTIALS + ND + 1;
constexpr size_t NOALLOC_SCRATCH_BYTES = NOALLOC_SCRATCH_DOUBLES * sizeof(double);
static_assert(NOALLOC_SCRATCH_BYTES == 94808, "scratch size stated in the header");

// The scratch. In host code this name is only a host-side stand-in, not a
// device address: kernels get the address from cudaGetSymbolAddress.
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

// Records the message for bgk_last_error() and returns the code.
int fail(int code, const char* msg) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "bgk_diagnostics_noalloc: %s", msg);
  set_last_error(buf);
  return code;
}

// Device address of the scratch in the current context, looked up on every
// call. The lookup is a host-side table query once the module is loaded in
// the context, so nothing is cached: a cached address would go stale after a
// cudaDeviceReset (the module is loaded again, possibly elsewhere) and would
// belong to the wrong context for a caller whose current context is not the
// device's primary one (one made through the driver API by another runtime).
// The first call in a context loads the module there, which is why that first
// call must come before any stream capture.
int scratch_in_current_context(double** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return fail(BGK_ERR_CUDA, cudaGetErrorString(e));
  if (!p) return fail(BGK_ERR_CUDA, "null scratch address");
  *out = (double*)p;
  return BGK_OK;
}

}  // namespace

extern "C" int bgk_diagnostics_noalloc(const void* const* pops19, int lx, int ly, int lz, int pitch_x, int precision,
                                       double svisc, double omega, double u0, double fp16_scale, int mode, int itime,
                                       bgk_diag* out, void* stream) {
  if (!pops19 || !out) return fail(BGK_ERR_INVALID, "null populations or output");
  for (int q = 0; q < Q; ++q)
    if (!pops19[q]) return fail(BGK_ERR_INVALID, "null population pointer");
  if (lx < 1 || ly < 1 || lz < 1 || pitch_x < lx) return fail(BGK_ERR_INVALID, "invalid box or row pitch");
  if ((long long)pitch_x * ly * lz >= (1LL << 31))
    return fail(BGK_ERR_INVALID, "box too large: pitch_x*ly*lz must stay below 2^31 cells per population");
  if (precision < BGK_FP64 || precision > BGK_FP16DEV) return fail(BGK_ERR_INVALID, "invalid precision");
  if (mode != BGK_CORRECTED && mode != BGK_FAITHFUL) return fail(BGK_ERR_INVALID, "invalid mode");
  double scale = 1.0;
  if (precision == BGK_FP16DEV) {
    int ex;
    if (!(fp16_scale > 0.0) || std::frexp(fp16_scale, &ex) != 0.5)
      return fail(BGK_ERR_INVALID, "fp16_scale must be a positive power of two");
    scale = fp16_scale;
  }
  double* scratch = nullptr;
  int rc = scratch_in_current_context(&scratch);
  if (rc) return rc;
  double* partials = scratch;
  double* totals = scratch + NOALLOC_PARTIALS;

  Lattice lat{};
  lat.form = precision;
  lat.g.nx = lx;
  lat.g.ny = ly;
  lat.g.nz = lz;
  lat.g.sx = pitch_x;
  lat.g.qs = 0;
  for (int q = 0; q < Q; ++q) lat.p[q] = const_cast<void*>(pops19[q]);
  cudaStream_t st = (cudaStream_t)stream;
  const bool faithful = mode == BGK_FAITHFUL;
  // Every partial slot and every total is written by these kernels before it
  // is read, so nothing left from an earlier call has to be cleared.
  cudaError_t e = launch_diag(lat, LAY_TWO, svisc, omega, scale, partials, nullptr, st);
  if (e == cudaSuccess) e = launch_finalize(partials, totals, st);
  if (e == cudaSuccess && faithful) e = launch_last_zj(lat, LAY_TWO, scale, totals + ND, st);
  double t[ND + 1] = {0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(t, totals, sizeof(t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(BGK_ERR_CUDA, cudaGetErrorString(e));

  const double N = (double)lx * ly * lz;
  out->itime = itime;
  out->rho_mean = t[0] / N;
  out->ux_mean = t[1] / N;
  out->uy_mean = t[2] / N;
  out->uz_mean = faithful ? (t[2] + t[ND]) / N : t[3] / N;
  out->ke_mean = t[4] / N;
  const float dxs = (2.0f * 3.141592f) / (float)lx;
  double u0r;
  if (precision == BGK_FP64) {
    volatile double dt = (double)dxs * u0;
    out->t = (double)(float)itime * dt;
    u0r = u0;
  } else {
    volatile float dt = dxs * (float)u0;
    volatile float tt = (float)itime * dt;
    out->t = (double)tt;
    u0r = (double)(float)u0;
  }
  out->tke = t[5];
  out->tke_norm = t[5] / (double)lx / (double)ly / (double)lz / (u0r * u0r);
  out->diss = t[6];
  out->eps_strain = t[7] / N;
  out->enstrophy = 0.0;  // needs a 3-component velocity field: not computed here
  out->nonfinite = (long long)t[8];
  if (out->nonfinite > 0) {
    char msg[160];
    std::snprintf(msg, sizeof(msg), "%lld cells with non-finite density or velocity at itime %d", out->nonfinite,
                  itime);
    return fail(BGK_ERR_NONFINITE, msg);
  }
  return BGK_OK;
}
