// C-ABI of the library (include/bgk3d.h): context, parameter checks, device
// memory, and the reference's call sequence mapped onto the kernels.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "bgk3d.h"
#include "kernels.h"

using namespace bgk;

namespace {

thread_local char g_err[512] = "";

void set_err(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int cuda_fail(cudaError_t e, const char* what) {
  set_err("%s: %s", what, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? BGK_ERR_NOMEM : BGK_ERR_CUDA;
}

#define CK(call)                                         \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

// Rows are padded to a multiple of 32 elements so that every row starts on a
// 64..256-byte boundary; populations start on 256-element boundaries.
constexpr int ROW_ALIGN = 32;
constexpr long long POP_ALIGN = 256;
// Staging for host velocity input: this many cells per chunk (whole planes).
// Cells per chunk of a velocity-field upload from host memory: two staging
// sets of three such chunks (96 MB) let the copy of one chunk run beside the
// initialisation kernel of the previous one.
constexpr long long INIT_CHUNK_CELLS = 1LL << 21;

}  // namespace

struct bgk_ctx {
  bgk_params p;
  int form = 0, scheme = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t mark = nullptr;  // bgk_record_event / bgk_wait_event
  // z-slab: second stream for the interior planes and its fork / join events
  cudaStream_t st_in = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // z-slab: timing events around the edge-plane kernel of each step
  cudaEvent_t ev_edge0 = nullptr, ev_edge1 = nullptr;
  int edge_timed = 0;
  // faithful two-lattice box: boundary planes of the states at the start of
  // the last two steps (by step parity) and the step each one holds
  void* faith_mem = nullptr;
  long long faith_step[2] = {-1, -1};
  Geo g{};
  size_t es = 8;
  void* memA = nullptr;
  void* memB = nullptr;
  Lattice A{}, B{};
  int lay = LAY_TWO;
  int initialized = 0;
  long long step = 0;
  double omega = 0.0, scale = 1.0;
  double* partials = nullptr;
  double* totals = nullptr;
  double* h_tot = nullptr;  // pinned
  unsigned int* d_max = nullptr;
  int* d_err = nullptr;     // set on the device when a pipelined kernel's wait ran out
  int* h_err = nullptr;     // pinned copy
  void* vel = nullptr;
  void* stage = nullptr;
  size_t stage_bytes = 0;
  // host upload pipeline: copy stream, staging set filled / free again
  cudaStream_t st_copy = nullptr;
  cudaEvent_t ev_full[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
  long long launches = 0;
  long long dev_bytes = 0;
  void* fft_buf = nullptr;
  size_t fft_bytes = 0;
  cufftHandle plan = 0;
  int plan_ok = 0;
  double* d_bins = nullptr;
  int nbins_alloc = 0;
  // adjoint / tangent buffers, kept for later calls (freed by bgk_destroy)
  std::vector<void*> lat_pool;   // lattice-sized blocks (Q * qs * es bytes)
  double* vel_pool[4] = {nullptr, nullptr, nullptr, nullptr};  // 3*N doubles each
  double* adj_acc = nullptr;
  long long adj_acc_n = 0;
  double* adj_tot = nullptr;
  size_t adj_cache_bytes = 0;  // bgk_adjoint_cache budget
  int adj_mode = BGK_ADJ_RECOMPUTE;  // bgk_adjoint_mode
  // z-slab (proc_z > 1): ghost buffer [parity 2][face 2][NZF][plane_elems],
  // the neighbours' buffers, and whether the neighbours' planes were filled
  // from the current state
  int slab = 0;
  void* halo_mem = nullptr;
  size_t halo_bytes = 0;
  long long plane_elems = 0;
  void* nb_below = nullptr;
  void* nb_above = nullptr;
  int primed = 0;
  std::vector<void*> ipc_maps;
};

namespace {

long long ncell(const bgk_ctx* c) { return (long long)c->g.nx * c->g.ny * c->g.nz; }
// cells of the whole box (all slabs)
double global_cells(const bgk_ctx* c) { return (double)c->g.nx * (double)c->g.ny * (double)c->g.gz; }

// Ghost-plane pointers of a slab: its own planes of parity rp (read) and the
// neighbours' planes of parity wp (written); face 0 is the plane below a
// slab (cz = +1 populations), face 1 the plane above (cz = -1).
SlabLinks slab_links(const bgk_ctx* c, int rp, int wp) {
  SlabLinks l{};
  auto plane = [&](void* base, int par, int face, int s) -> void* {
    if (!base) return nullptr;
    return (char*)base + (size_t)(((par * 2 + face) * NZF + s) * c->plane_elems) * c->es;
  };
  for (int s = 0; s < NZF; ++s) {
    l.in_lo[s] = plane(c->halo_mem, rp, 0, s);
    l.in_hi[s] = plane(c->halo_mem, rp, 1, s);
    l.up[s] = plane(c->nb_above, wp, 0, s);
    l.dn[s] = plane(c->nb_below, wp, 1, s);
  }
  return l;
}
size_t rsize(const bgk_ctx* c) { return c->form == FORM_F64 ? 8 : 4; }

int dev_alloc(bgk_ctx* c, void** ptr, size_t bytes, const char* what) {
  cudaError_t e = cudaMalloc(ptr, bytes);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    *ptr = nullptr;
    set_err("cudaMalloc(%zu bytes) for %s: %s", bytes, what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? BGK_ERR_NOMEM : BGK_ERR_CUDA;
  }
  c->dev_bytes += (long long)bytes;
  return BGK_OK;
}

int ensure_stage(bgk_ctx* c, size_t bytes) {
  if (c->stage_bytes >= bytes) return BGK_OK;
  if (c->stage) {
    CK(cudaStreamSynchronize(c->st));
    cudaFree(c->stage);
    c->dev_bytes -= (long long)c->stage_bytes;
    c->stage = nullptr;
    c->stage_bytes = 0;
  }
  int rc = dev_alloc(c, &c->stage, bytes, "staging buffer");
  if (rc) return rc;
  c->stage_bytes = bytes;
  return BGK_OK;
}

int ensure_vel(bgk_ctx* c) {
  if (c->vel) return BGK_OK;
  return dev_alloc(c, &c->vel, 3 * (size_t)ncell(c) * rsize(c), "velocity field");
}

int check_ctx(const bgk_ctx* c) {
  if (!c) {
    set_err("null context");
    return BGK_ERR_INVALID;
  }
  return BGK_OK;
}

int check_init(bgk_ctx* c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!c->initialized) {
    set_err("populations not initialised (call bgk_init_tgv, bgk_init_velocity or bgk_put_populations)");
    return BGK_ERR_STATE;
  }
  return BGK_OK;
}

// omega = (uno+uno)/((6.0*svisc)+1.0), SRC/hencol.F90:31, in the arithmetic
// type of the form (volatile keeps each rounding as written).
double omega_of(const bgk_params& p, int form) {
  if (p.use_omega) return p.omega;
  if (form == FORM_F64) {
    volatile double s = p.svisc;
    volatile double a = 6.0 * s;
    volatile double b = a + 1.0;
    return (1.0 + 1.0) / b;
  }
  volatile float s = (float)p.svisc;
  volatile float a = 6.0f * s;
  volatile float b = a + 1.0f;
  volatile float o = (1.0f + 1.0f) / b;
  return (double)o;
}

// Smallest-exponent-headroom scale for the FP16 form:
// 2^floor(log2(65504 / (4 max|f - w|))).
double fp16_scale_for(float maxabs) {
  if (!(maxabs > 0.f) || !std::isfinite(maxabs)) return 1.0;
  const double r = 65504.0 / (4.0 * (double)maxabs);
  return std::ldexp(1.0, (int)std::floor(std::log2(r)));
}

int set_scale_from_max(bgk_ctx* c) {
  unsigned int bits = 0;
  CK(cudaMemcpyAsync(&bits, c->d_max, sizeof(bits), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  float m;
  std::memcpy(&m, &bits, sizeof(m));
  c->scale = fp16_scale_for(m);
  return BGK_OK;
}

int init_layout(const bgk_ctx* c) { return c->scheme == BGK_AA ? LAY_AAE : LAY_TWO; }

// Synchronises the stream and reports a bounded wait of a pipelined kernel
// that ran out (the step it belonged to did not complete).
int sync_and_check(bgk_ctx* c) {
  CK(cudaMemcpyAsync(c->h_err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (*c->h_err) {
    set_err("a stream-collide step gave up waiting for its row copies; populations are invalid");
    return BGK_ERR_CUDA;
  }
  return BGK_OK;
}

// Equilibrium initial condition from a velocity field: host arrays go
// through a staging buffer in chunks of whole planes; device arrays (on the
// context's device) are read in place, chunk by chunk in the same order.
int init_velocity_impl(bgk_ctx* c, const double* u, const double* v, const double* w, double rho, bool on_device) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!u || !v || !w) {
    set_err("null velocity array");
    return BGK_ERR_INVALID;
  }
  if (!(rho > 0.0) || !std::isfinite(rho)) {
    set_err("rho must be positive and finite, got %g", rho);
    return BGK_ERR_INVALID;
  }
  CK(cudaSetDevice(c->p.device));
  if (on_device) {
    for (const double* p : {u, v, w}) {
      cudaPointerAttributes at{};
      CK(cudaPointerGetAttributes(&at, p));
      if ((at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) || at.device != c->p.device) {
        set_err("velocity arrays must be device memory of device %d", c->p.device);
        return BGK_ERR_INVALID;
      }
    }
  }
  const long long plane = (long long)c->g.nx * c->g.ny;
  int nk = (int)(INIT_CHUNK_CELLS / plane);
  if (nk < 1) nk = 1;
  if (nk > c->g.nz) nk = c->g.nz;
  const size_t chunk = (size_t)plane * nk;
  double *su = nullptr, *sv = nullptr, *sw = nullptr;
  if (!on_device) {
    // two staging sets of three chunks; the copies run on their own stream
    rc = ensure_stage(c, 2 * 3 * chunk * sizeof(double));
    if (rc) return rc;
    if (!c->st_copy) CK(cudaStreamCreateWithFlags(&c->st_copy, cudaStreamNonBlocking));
    for (int b = 0; b < 2; ++b) {
      if (!c->ev_full[b]) CK(cudaEventCreateWithFlags(&c->ev_full[b], cudaEventDisableTiming));
      if (!c->ev_free[b]) CK(cudaEventCreateWithFlags(&c->ev_free[b], cudaEventDisableTiming));
    }
    // nothing queued on the context's stream before this call may still
    // read a staging set when the first copies land
    CK(cudaEventRecord(c->ev_free[0], c->st));
    CK(cudaEventRecord(c->ev_free[1], c->st));
  }
  const int lay = init_layout(c);
  const bool measure = c->form == FORM_F16 && c->p.fp16_scale == 0.0;
  if (measure) CK(cudaMemsetAsync(c->d_max, 0, sizeof(unsigned int), c->st));
  for (int pass = measure ? 0 : 1; pass < 2; ++pass) {
    if (pass == 1 && measure) {
      rc = set_scale_from_max(c);
      if (rc) return rc;
    }
    int set = 0;  // staging set of this chunk
    for (int k0 = 0; k0 < c->g.nz; k0 += nk, set ^= 1) {
      const int nkk = k0 + nk <= c->g.nz ? nk : c->g.nz - k0;
      const size_t off = (size_t)plane * k0, cnt = (size_t)plane * nkk * sizeof(double);
      if (on_device) {
        su = const_cast<double*>(u) + off;
        sv = const_cast<double*>(v) + off;
        sw = const_cast<double*>(w) + off;
      } else {
        // copy into this set once the kernel that read it two chunks ago is
        // done, while the context's stream initialises the previous chunk
        su = (double*)c->stage + (size_t)set * 3 * chunk;
        sv = su + chunk;
        sw = sv + chunk;
        CK(cudaStreamWaitEvent(c->st_copy, c->ev_free[set], 0));
        CK(cudaMemcpyAsync(su, u + off, cnt, cudaMemcpyHostToDevice, c->st_copy));
        CK(cudaMemcpyAsync(sv, v + off, cnt, cudaMemcpyHostToDevice, c->st_copy));
        CK(cudaMemcpyAsync(sw, w + off, cnt, cudaMemcpyHostToDevice, c->st_copy));
        CK(cudaEventRecord(c->ev_full[set], c->st_copy));
        CK(cudaStreamWaitEvent(c->st, c->ev_full[set], 0));
      }
      CK(launch_init_velocity(c->A, lay, su, sv, sw, rho, k0, nkk, pass == 0 ? 1.0 : c->scale,
                              pass == 0 ? c->d_max : nullptr, c->st));
      if (!on_device) CK(cudaEventRecord(c->ev_free[set], c->st));
      c->launches++;
    }
  }
  CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st));
  CK(cudaStreamSynchronize(c->st));
  c->lay = lay;
  c->step = 0;
  c->initialized = 1;
  c->faith_step[0] = c->faith_step[1] = -1;
  c->primed = 0;
  return BGK_OK;
}

// Faithful mode on a whole two-lattice box reproduces the ghost cells the
// reference's dissipation pulls from: it runs after col_MC's pointer swap
// (SRC/col_MC.F90:364-421, SRC/dissipation.F90:76-94), so after step t the
// current lattice's ghosts hold the periodic images of the state at the
// start of step t - 1 (its boundaries call), and after step 1 they were
// never written (zero deviations, as a freshly allocated lattice). The
// boundary planes of each step's starting state are kept by step parity.
bool faith_on(const bgk_ctx* c) {
  return c->p.mode == BGK_FAITHFUL && c->scheme == BGK_TWO_LATTICE && !c->slab;
}

void* faith_buf(const bgk_ctx* c, long long step) {
  return (char*)c->faith_mem + (size_t)(step & 1) * (size_t)faith_planes_elems(c->g) * c->es;
}

int faith_snapshot(bgk_ctx* c) {
  if (!faith_on(c)) return BGK_OK;
  if (!c->faith_mem) {
    int rc = dev_alloc(c, &c->faith_mem, 2 * (size_t)faith_planes_elems(c->g) * c->es, "faithful-mode ghost planes");
    if (rc) return rc;
  }
  CK(launch_faith_snapshot(c->A, faith_buf(c, c->step), c->st));
  c->launches++;
  c->faith_step[c->step & 1] = c->step;
  return BGK_OK;
}

int compute_diag(bgk_ctx* c, int itime, bgk_diag* out, int want_extras) {
  const bool extras = want_extras && c->p.extras && !c->slab;
  if (extras) {
    int rc = ensure_vel(c);
    if (rc) return rc;
  }
  const SlabLinks hl = c->slab ? slab_links(c, (int)(c->step & 1), 0) : SlabLinks{};
  const void* faith = nullptr;
  bool faith_zero = false;
  if (faith_on(c) && c->step == 1) {
    faith_zero = true;
  } else if (faith_on(c) && c->step >= 2 && c->faith_step[c->step & 1] == c->step - 2) {
    faith = faith_buf(c, c->step);
  }
  CK(launch_diag(c->A, c->lay, c->p.svisc, c->omega, c->scale, c->partials, extras ? c->vel : nullptr, c->st,
                 c->slab ? &hl : nullptr, faith, faith_zero));
  c->launches++;
  if (extras) {
    CK(launch_enstrophy(c->A, c->vel, c->partials, c->st));
    c->launches++;
  }
  CK(launch_finalize(c->partials, c->totals, c->st));
  c->launches++;
  const bool faithful = c->p.mode == BGK_FAITHFUL;
  if (faithful) {
    CK(launch_last_zj(c->A, c->lay, c->scale, c->totals + ND, c->st));
    c->launches++;
  }
  CK(cudaMemcpyAsync(c->h_tot, c->totals, (ND + 1) * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  int rc = sync_and_check(c);
  if (rc) return rc;
  const double* t = c->h_tot;
  // a z-slab returns its contribution to the global means
  const double N = global_cells(c);
  out->itime = itime;
  out->rho_mean = t[0] / N;
  out->ux_mean = t[1] / N;
  out->uy_mean = t[2] / N;
  // SRC/diagno.F90:110 accumulates ztot = ytot + zj: the final value is the
  // full y sum plus zj of the last cell.
  out->uz_mean = faithful ? (t[2] + t[ND]) / N : t[3] / N;
  out->ke_mean = t[4] / N;
  // t = float(itime)*dt with dx = (2.0*3.141592)/float(lx) in single precision
  // and dt = dx*u0 (SRC/dissipation.F90:65-66,262), in the form's arithmetic.
  const float dxs = (2.0f * 3.141592f) / (float)c->g.nx;
  double u0r;
  if (c->form == FORM_F64) {
    volatile double dt = (double)dxs * c->p.u0;
    out->t = (double)(float)itime * dt;
    u0r = c->p.u0;
  } else {
    volatile float dt = dxs * (float)c->p.u0;
    volatile float tt = (float)itime * dt;
    out->t = (double)tt;
    u0r = (double)(float)c->p.u0;
  }
  out->tke = t[5];
  out->tke_norm = t[5] / (double)c->g.nx / (double)c->g.ny / (double)c->g.gz / (u0r * u0r);
  out->diss = t[6];
  out->eps_strain = t[7] / N;
  out->nonfinite = (long long)t[8];
  out->enstrophy = extras ? t[9] / N : 0.0;
  if (out->nonfinite > 0) {
    set_err("diagnostics: %lld cells with non-finite density or velocity at itime %d", out->nonfinite, itime);
    return BGK_ERR_NONFINITE;
  }
  return BGK_OK;
}

}  // namespace

void bgk::set_last_error(const char* msg) { set_err("%s", msg); }

extern "C" {

int bgk_params_default(bgk_params* p) {
  if (!p) return BGK_ERR_INVALID;
  std::memset(p, 0, sizeof(*p));
  p->lx = p->ly = p->lz = 64;
  p->svisc = 0.01;
  p->u0 = 0.05;
  p->precision = BGK_FP64;
  p->scheme = BGK_TWO_LATTICE;
  p->icheck = 10;
  p->mode = BGK_CORRECTED;
  p->fp16_scale = 0.0;
  p->device = 0;
  p->use_omega = 0;
  p->omega = 0.0;
  p->extras = 1;
  p->kernel = 0;
  p->les_cs = 0.0;
  p->proc_z = 1;
  p->coord_z = 0;
  return BGK_OK;
}

int bgk_create(const bgk_params* p, bgk_ctx** out) {
  if (!p || !out) {
    set_err("null argument");
    return BGK_ERR_INVALID;
  }
  *out = nullptr;
  // parameter checks (the reference stops on inconsistent sizes,
  // SRC/input.F90:66-82; here every check returns an error instead)
  if (p->proc_z < 1 || p->coord_z < 0 || p->coord_z >= p->proc_z) {
    set_err("invalid z decomposition: proc_z %d, coord_z %d", p->proc_z, p->coord_z);
    return BGK_ERR_INVALID;
  }
  if (p->lx < 1 || p->ly < 1 || p->lz < 1 || p->lz % p->proc_z != 0 || p->lz / p->proc_z > 65535) {
    set_err("invalid box %d x %d x %d for %d z-slab(s)", p->lx, p->ly, p->lz, p->proc_z);
    return BGK_ERR_INVALID;
  }
  const int nzl = p->lz / p->proc_z;  // planes of this context
  if (p->precision < BGK_FP64 || p->precision > BGK_FP16DEV) {
    set_err("invalid precision %d", p->precision);
    return BGK_ERR_INVALID;
  }
  if (p->scheme != BGK_TWO_LATTICE && p->scheme != BGK_AA) {
    set_err("invalid scheme %d", p->scheme);
    return BGK_ERR_INVALID;
  }
  if (p->mode != BGK_CORRECTED && p->mode != BGK_FAITHFUL) {
    set_err("invalid mode %d", p->mode);
    return BGK_ERR_INVALID;
  }
  if (p->proc_z > 1 && (p->scheme != BGK_TWO_LATTICE || p->mode != BGK_CORRECTED ||
                        (p->precision == BGK_FP16DEV && p->fp16_scale == 0.0))) {
    set_err("z-slabs run the two-lattice scheme in corrected mode, FP16 with an explicit fp16_scale");
    return BGK_ERR_INVALID;
  }
  if (p->kernel != 0 && p->kernel != 1 && p->kernel != 2 && p->kernel != 4 && p->kernel != 8) {
    set_err("kernel must be 0, 1, 2, 4 or 8 (got %d)", p->kernel);
    return BGK_ERR_INVALID;
  }
  if (!(p->les_cs >= 0.0 && p->les_cs <= 10.0)) {
    set_err("les_cs must be a Smagorinsky constant in [0, 10] (got %g)", p->les_cs);
    return BGK_ERR_INVALID;
  }
  if (p->icheck < 1) {
    set_err("icheck must be >= 1 (got %d)", p->icheck);
    return BGK_ERR_INVALID;
  }
  if (p->use_omega) {
    if (!(p->omega >= 0.0 && p->omega <= 2.0)) {
      set_err("omega override %g outside [0, 2]", p->omega);
      return BGK_ERR_INVALID;
    }
  } else if (!(p->svisc > 0.0) || !std::isfinite(p->svisc)) {
    set_err("svisc must be > 0 (tau = 3 svisc + 1/2 > 1/2), got %g", p->svisc);
    return BGK_ERR_INVALID;
  }
  if (!std::isfinite(p->u0)) {
    set_err("u0 must be finite");
    return BGK_ERR_INVALID;
  }
  if (p->fp16_scale != 0.0) {
    int ex;
    const double m = std::frexp(p->fp16_scale, &ex);
    if (!(p->fp16_scale > 0.0) || m != 0.5) {
      set_err("fp16_scale must be 0 or a positive power of two, got %g", p->fp16_scale);
      return BGK_ERR_INVALID;
    }
  }
  const long long sx = ((long long)p->lx + ROW_ALIGN - 1) / ROW_ALIGN * ROW_ALIGN;
  const long long cells = sx * p->ly * nzl;
  if (cells >= (1LL << 31) - POP_ALIGN) {
    set_err("box too large: %lld padded cells per population (limit 2^31)", cells);
    return BGK_ERR_INVALID;
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    set_err("no CUDA device: %s", cudaGetErrorString(e));
    return BGK_ERR_CUDA;
  }
  if (p->device < 0 || p->device >= ndev) {
    set_err("device %d out of range (%d devices)", p->device, ndev);
    return BGK_ERR_INVALID;
  }
  CK(cudaSetDevice(p->device));

  bgk_ctx* c = new bgk_ctx();
  c->p = *p;
  c->form = p->precision;
  c->scheme = p->scheme;
  c->es = c->form == FORM_F64 ? 8 : (c->form == FORM_F32 ? 4 : 2);
  c->g.nx = p->lx;
  c->g.ny = p->ly;
  c->g.nz = nzl;
  c->g.sx = (int)sx;
  c->g.qs = (cells + POP_ALIGN - 1) / POP_ALIGN * POP_ALIGN;
  c->g.z0 = p->coord_z * nzl;
  c->g.gz = p->lz;
  c->slab = p->proc_z > 1;
  c->omega = omega_of(*p, c->form);
  c->scale = c->form == FORM_F16 ? (p->fp16_scale != 0.0 ? p->fp16_scale : 1.0) : 1.0;
  c->A.form = c->B.form = c->form;
  c->A.g = c->B.g = c->g;

  auto fail = [&](int rc) {
    bgk_destroy(c);
    return rc;
  };
  e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(cuda_fail(e, "cudaStreamCreate"));
  const size_t pop_bytes = (size_t)c->g.qs * c->es;
  int rc = dev_alloc(c, &c->memA, Q * pop_bytes, "lattice a");
  if (rc) return fail(rc);
  for (int q = 0; q < Q; ++q) c->A.p[q] = (char*)c->memA + q * pop_bytes;
  if (c->scheme == BGK_TWO_LATTICE) {
    // b01..b18; b19 is never used (pop 19 is updated in place,
    // SRC/col_MC.F90:351), so it is not allocated
    rc = dev_alloc(c, &c->memB, (Q - 1) * pop_bytes, "lattice b");
    if (rc) return fail(rc);
    for (int q = 0; q < Q - 1; ++q) c->B.p[q] = (char*)c->memB + q * pop_bytes;
    c->B.p[Q - 1] = c->A.p[Q - 1];
  }
  rc = dev_alloc(c, (void**)&c->partials, (size_t)DIAG_BLOCKS * ND * 2 * sizeof(double), "diagnostic partials");
  if (rc) return fail(rc);
  rc = dev_alloc(c, (void**)&c->totals, (ND + 1) * sizeof(double), "diagnostic totals");
  if (rc) return fail(rc);
  rc = dev_alloc(c, (void**)&c->d_max, sizeof(unsigned int), "scale probe");
  if (rc) return fail(rc);
  rc = dev_alloc(c, (void**)&c->d_err, sizeof(int), "error flag");
  if (rc) return fail(rc);
  e = cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st);
  if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMemset"));
  e = cudaMallocHost((void**)&c->h_err, sizeof(int));
  if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMallocHost"));
  c->A.err = c->B.err = c->d_err;
  e = cudaMallocHost((void**)&c->h_tot, (ND + 1) * sizeof(double));
  if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMallocHost"));
  if (c->slab) {
    c->plane_elems = (sx * p->ly + POP_ALIGN - 1) / POP_ALIGN * POP_ALIGN;
    c->halo_bytes = (size_t)(2 * 2 * NZF) * (size_t)c->plane_elems * c->es;
    rc = dev_alloc(c, &c->halo_mem, c->halo_bytes, "ghost planes");
    if (rc) return fail(rc);
    e = cudaStreamCreateWithFlags(&c->st_in, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev_edge0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev_edge1);
    if (e != cudaSuccess) return fail(cuda_fail(e, "slab stream"));
    e = cudaMemsetAsync(c->halo_mem, 0, c->halo_bytes, c->st);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMemset"));
  }
  c->lay = init_layout(c);
  *out = c;
  return BGK_OK;
}

int bgk_destroy(bgk_ctx* c) {
  if (!c) return BGK_OK;
  cudaSetDevice(c->p.device);
  if (c->st_in) cudaStreamSynchronize(c->st_in);
  if (c->st) cudaStreamSynchronize(c->st);
  if (c->plan_ok) cufftDestroy(c->plan);
  cudaFree(c->memA);
  cudaFree(c->memB);
  cudaFree(c->partials);
  cudaFree(c->totals);
  cudaFree(c->d_max);
  cudaFree(c->d_err);
  if (c->h_err) cudaFreeHost(c->h_err);
  cudaFree(c->vel);
  cudaFree(c->stage);
  cudaFree(c->fft_buf);
  cudaFree(c->d_bins);
  for (void* m : c->lat_pool) cudaFree(m);
  for (void* m : c->ipc_maps) cudaIpcCloseMemHandle(m);
  cudaFree(c->halo_mem);
  cudaFree(c->faith_mem);
  for (double* m : c->vel_pool) cudaFree(m);
  cudaFree(c->adj_acc);
  cudaFree(c->adj_tot);
  if (c->h_tot) cudaFreeHost(c->h_tot);
  if (c->mark) cudaEventDestroy(c->mark);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->ev_edge0) cudaEventDestroy(c->ev_edge0);
  if (c->ev_edge1) cudaEventDestroy(c->ev_edge1);
  for (int b = 0; b < 2; ++b) {
    if (c->ev_full[b]) cudaEventDestroy(c->ev_full[b]);
    if (c->ev_free[b]) cudaEventDestroy(c->ev_free[b]);
  }
  if (c->st_copy) cudaStreamDestroy(c->st_copy);
  if (c->st_in) cudaStreamDestroy(c->st_in);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return BGK_OK;
}

int bgk_init_tgv(bgk_ctx* c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  CK(cudaSetDevice(c->p.device));
  const int lay = init_layout(c);
  const int faithful = c->p.mode == BGK_FAITHFUL;
  if (c->form == FORM_F16 && c->p.fp16_scale == 0.0) {
    CK(cudaMemsetAsync(c->d_max, 0, sizeof(unsigned int), c->st));
    CK(launch_init_tgv(c->A, lay, c->p.u0, faithful, 1.0, c->d_max, c->st));
    c->launches++;
    rc = set_scale_from_max(c);
    if (rc) return rc;
  }
  CK(launch_init_tgv(c->A, lay, c->p.u0, faithful, c->scale, nullptr, c->st));
  c->launches++;
  CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st));
  c->lay = lay;
  c->step = 0;
  c->initialized = 1;
  c->faith_step[0] = c->faith_step[1] = -1;
  c->primed = 0;
  return BGK_OK;
}

int bgk_init_velocity(bgk_ctx* c, const double* u, const double* v, const double* w, double rho) {
  return init_velocity_impl(c, u, v, w, rho, false);
}

int bgk_init_velocity_device(bgk_ctx* c, const double* u, const double* v, const double* w, double rho) {
  return init_velocity_impl(c, u, v, w, rho, true);
}

int bgk_boundaries(bgk_ctx* c, int itime) {
  (void)itime;
  return check_ctx(c);
}

int bgk_col_mc(bgk_ctx* c, int itime) {
  (void)itime;
  int rc = check_init(c);
  if (rc) return rc;
  CK(cudaSetDevice(c->p.device));
  if (c->slab && (!c->nb_below || !c->nb_above || !c->primed)) {
    set_err("z-slab: call bgk_halo_connect and then bgk_halo_prime (after every new state) before stepping");
    return BGK_ERR_STATE;
  }
  if (c->slab) {
    // boundary planes on the context's stream, interior planes side by side on
    // the second one; the join puts everything later on the context's stream
    // behind both
    const SlabLinks l = slab_links(c, (int)(c->step & 1), (int)((c->step + 1) & 1));
    CK(cudaEventRecord(c->ev_fork, c->st));
    CK(cudaStreamWaitEvent(c->st_in, c->ev_fork, 0));
    // the edge-plane kernel is the only work on st between these two events
    CK(cudaEventRecord(c->ev_edge0, c->st));
    CK(launch_slab(c->A, c->B, l, c->omega, c->scale, c->p.les_cs, c->st, c->st_in));
    CK(cudaEventRecord(c->ev_edge1, c->st));
    c->edge_timed = 1;
    CK(cudaEventRecord(c->ev_join, c->st_in));
    CK(cudaStreamWaitEvent(c->st, c->ev_join, 0));
    if (c->g.nz > 2) c->launches++;  // edge planes and interior are two launches
  } else if (c->scheme == BGK_TWO_LATTICE) {
    rc = faith_snapshot(c);
    if (rc) return rc;
    CK(launch_two_lattice(c->A, c->B, c->omega, c->scale, c->p.les_cs, c->p.kernel, c->st));
  }
  if (c->scheme == BGK_TWO_LATTICE) {
    // pointer swap of pops 01..18, SRC/col_MC.F90:364-421
    for (int q = 0; q < Q - 1; ++q) {
      void* t = c->A.p[q];
      c->A.p[q] = c->B.p[q];
      c->B.p[q] = t;
    }
  } else {
    const int odd = c->lay == LAY_AAE;
    CK(launch_aa(c->A, odd, c->omega, c->scale, c->p.les_cs, c->p.kernel, c->st));
    c->lay = odd ? LAY_AAN : LAY_AAE;
  }
  c->launches++;
  c->step++;
  c->A.stall = c->B.stall = 0;
  return BGK_OK;
}

int bgk_halo_buffer(const bgk_ctx* c, void** dptr, size_t* bytes) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!dptr || !bytes || !c->slab) {
    set_err("bgk_halo_buffer: null argument or not a z-slab context (proc_z = 1)");
    return BGK_ERR_INVALID;
  }
  *dptr = c->halo_mem;
  *bytes = c->halo_bytes;
  return BGK_OK;
}

int bgk_halo_ipc_handle(const bgk_ctx* c, void* handle64) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!handle64 || !c->slab) {
    set_err("bgk_halo_ipc_handle: null argument or not a z-slab context");
    return BGK_ERR_INVALID;
  }
  static_assert(sizeof(cudaIpcMemHandle_t) == 64, "IPC handle size");
  CK(cudaSetDevice(c->p.device));
  cudaIpcMemHandle_t h;
  CK(cudaIpcGetMemHandle(&h, c->halo_mem));
  std::memcpy(handle64, &h, 64);
  return BGK_OK;
}

int bgk_halo_ipc_open(bgk_ctx* c, const void* handle64, void** dptr) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!handle64 || !dptr || !c->slab) {
    set_err("bgk_halo_ipc_open: null argument or not a z-slab context");
    return BGK_ERR_INVALID;
  }
  CK(cudaSetDevice(c->p.device));
  cudaIpcMemHandle_t h;
  std::memcpy(&h, handle64, 64);
  void* p = nullptr;
  CK(cudaIpcOpenMemHandle(&p, h, cudaIpcMemLazyEnablePeerAccess));
  c->ipc_maps.push_back(p);
  *dptr = p;
  return BGK_OK;
}

int bgk_halo_connect(bgk_ctx* c, void* below, void* above) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!below || !above || !c->slab) {
    set_err("bgk_halo_connect: null buffer or not a z-slab context");
    return BGK_ERR_INVALID;
  }
  CK(cudaSetDevice(c->p.device));
  for (void* p : {below, above}) {
    cudaPointerAttributes a{};
    CK(cudaPointerGetAttributes(&a, p));
    if (a.type != cudaMemoryTypeDevice) {
      set_err("bgk_halo_connect: %p is not device memory", p);
      return BGK_ERR_INVALID;
    }
    if (a.device != c->p.device) {
      int ok = 0;
      CK(cudaDeviceCanAccessPeer(&ok, c->p.device, a.device));
      if (!ok) {
        set_err("bgk_halo_connect: device %d cannot access device %d", c->p.device, a.device);
        return BGK_ERR_INVALID;
      }
      cudaError_t e = cudaDeviceEnablePeerAccess(a.device, 0);
      if (e == cudaErrorPeerAccessAlreadyEnabled) (void)cudaGetLastError();
      else if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceEnablePeerAccess");
    }
  }
  c->nb_below = below;
  c->nb_above = above;
  c->primed = 0;
  return BGK_OK;
}

int bgk_slab_edge_time(bgk_ctx* c, double* us) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!us || !c->slab) {
    set_err("bgk_slab_edge_time: null argument or not a z-slab context");
    return BGK_ERR_INVALID;
  }
  if (!c->edge_timed) {
    set_err("bgk_slab_edge_time: no step has run on this slab yet");
    return BGK_ERR_STATE;
  }
  CK(cudaSetDevice(c->p.device));
  CK(cudaEventSynchronize(c->ev_edge1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c->ev_edge0, c->ev_edge1));
  *us = 1e3 * (double)ms;
  return BGK_OK;
}

int bgk_halo_prime(bgk_ctx* c) {
  int rc = check_init(c);
  if (rc) return rc;
  if (!c->slab || !c->nb_below || !c->nb_above) {
    set_err("bgk_halo_prime: not a connected z-slab context");
    return BGK_ERR_STATE;
  }
  CK(cudaSetDevice(c->p.device));
  const SlabLinks l = slab_links(c, 0, (int)(c->step & 1));
  CK(launch_halo_prime(c->A, l, c->st));
  c->launches++;
  c->primed = 1;
  return BGK_OK;
}

int bgk_debug_stall_next_step(bgk_ctx* c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (c->p.kernel != 8 || c->p.les_cs > 0.0 || c->slab) {
    set_err("bgk_debug_stall_next_step needs the row-pipelined kernel (params.kernel = 8, BGK collision)");
    return BGK_ERR_INVALID;
  }
  c->A.stall = c->B.stall = 1;
  return BGK_OK;
}

int bgk_run(bgk_ctx* c, int nsteps) {
  if (nsteps < 0) {
    set_err("nsteps < 0");
    return BGK_ERR_INVALID;
  }
  if (c && c->slab && nsteps > 1) {
    set_err("z-slab: one step per call, with the slabs synchronised between steps");
    return BGK_ERR_INVALID;
  }
  for (int s = 0; s < nsteps; ++s) {
    int rc = bgk_boundaries(c, (int)(c ? c->step + 1 : 0));
    if (rc) return rc;
    rc = bgk_col_mc(c, (int)(c->step + 1));
    if (rc) return rc;
  }
  return BGK_OK;
}

int bgk_diagnostic(bgk_ctx* c, int itime, bgk_diag* out) {
  int rc = check_init(c);
  if (rc) return rc;
  if (!out) {
    set_err("null output");
    return BGK_ERR_INVALID;
  }
  if (itime % c->p.icheck != 0) return BGK_SKIPPED;  // SRC/diagnostic.F90:37
  CK(cudaSetDevice(c->p.device));
  return compute_diag(c, itime, out, 1);
}

int bgk_diagno(bgk_ctx* c, int itime, double* o) {
  int rc = check_init(c);
  if (rc) return rc;
  if (!o) return BGK_ERR_INVALID;
  CK(cudaSetDevice(c->p.device));
  bgk_diag d;
  rc = compute_diag(c, itime, &d, 0);
  if (rc && rc != BGK_ERR_NONFINITE) return rc;
  o[0] = d.rho_mean; o[1] = d.ux_mean; o[2] = d.uy_mean; o[3] = d.uz_mean; o[4] = d.ke_mean;
  return rc;
}

int bgk_dissipation(bgk_ctx* c, int itime, double* o) {
  int rc = check_init(c);
  if (rc) return rc;
  if (!o) return BGK_ERR_INVALID;
  CK(cudaSetDevice(c->p.device));
  bgk_diag d;
  rc = compute_diag(c, itime, &d, 0);
  if (rc && rc != BGK_ERR_NONFINITE) return rc;
  o[0] = d.t; o[1] = d.tke_norm; o[2] = d.diss; o[3] = d.tke;
  return rc;
}

int bgk_get_populations(bgk_ctx* c, void* host) {
  int rc = check_init(c);
  if (rc) return rc;
  if (!host) return BGK_ERR_INVALID;
  CK(cudaSetDevice(c->p.device));
  const size_t n = (size_t)ncell(c);
  rc = ensure_stage(c, n * 8);
  if (rc) return rc;
  for (int q = 0; q < Q; ++q) {
    CK(launch_export(c->A, c->lay, q, c->stage, nullptr, c->scale, c->st));
    c->launches++;
    CK(cudaMemcpyAsync((char*)host + q * n * c->es, c->stage, n * c->es, cudaMemcpyDeviceToHost, c->st));
  }
  return sync_and_check(c);
}

int bgk_get_deviations(bgk_ctx* c, double* host) {
  int rc = check_init(c);
  if (rc) return rc;
  if (!host) return BGK_ERR_INVALID;
  CK(cudaSetDevice(c->p.device));
  const size_t n = (size_t)ncell(c);
  rc = ensure_stage(c, n * 8);
  if (rc) return rc;
  for (int q = 0; q < Q; ++q) {
    CK(launch_export(c->A, c->lay, q, nullptr, (double*)c->stage, c->scale, c->st));
    c->launches++;
    CK(cudaMemcpyAsync(host + q * n, c->stage, n * 8, cudaMemcpyDeviceToHost, c->st));
  }
  return sync_and_check(c);
}

int bgk_put_populations(bgk_ctx* c, const void* host) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!host) return BGK_ERR_INVALID;
  CK(cudaSetDevice(c->p.device));
  const size_t n = (size_t)ncell(c);
  rc = ensure_stage(c, n * 8);
  if (rc) return rc;
  const int lay = c->initialized ? c->lay : init_layout(c);
  for (int q = 0; q < Q; ++q) {
    CK(cudaMemcpyAsync(c->stage, (const char*)host + q * n * c->es, n * c->es, cudaMemcpyHostToDevice, c->st));
    CK(launch_import(c->A, lay, q, c->stage, c->st));
    c->launches++;
  }
  CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st));
  CK(cudaStreamSynchronize(c->st));
  c->lay = lay;
  if (!c->initialized) c->step = 0;
  c->initialized = 1;
  c->faith_step[0] = c->faith_step[1] = -1;
  c->primed = 0;
  return BGK_OK;
}

int bgk_get_velocity(bgk_ctx* c, double* u, double* v, double* w) {
  int rc = check_init(c);
  if (rc) return rc;
  if (!u || !v || !w) return BGK_ERR_INVALID;
  CK(cudaSetDevice(c->p.device));
  rc = ensure_vel(c);
  if (rc) return rc;
  CK(launch_diag(c->A, c->lay, c->p.svisc, c->omega, c->scale, c->partials, c->vel, c->st));
  c->launches++;
  const size_t n = (size_t)ncell(c);
  double* dst[3] = {u, v, w};
  if (c->form == FORM_F64) {
    for (int d = 0; d < 3; ++d)
      CK(cudaMemcpyAsync(dst[d], (double*)c->vel + d * n, n * 8, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  } else {
    std::vector<float> tmp(n);
    for (int d = 0; d < 3; ++d) {
      CK(cudaMemcpyAsync(tmp.data(), (float*)c->vel + d * n, n * 4, cudaMemcpyDeviceToHost, c->st));
      CK(cudaStreamSynchronize(c->st));
      for (size_t s = 0; s < n; ++s) dst[d][s] = (double)tmp[s];
    }
  }
  return BGK_OK;
}

int bgk_spectrum(bgk_ctx* c, int nbins, double* ek) {
  int rc = check_init(c);
  if (rc) return rc;
  if (c->slab) {
    set_err("bgk_spectrum needs the whole box (proc_z = 1)");
    return BGK_ERR_INVALID;
  }
  if (!ek || nbins < 1) {
    set_err("bgk_spectrum: invalid argument");
    return BGK_ERR_INVALID;
  }
  CK(cudaSetDevice(c->p.device));
  rc = ensure_vel(c);
  if (rc) return rc;
  CK(launch_diag(c->A, c->lay, c->p.svisc, c->omega, c->scale, c->partials, c->vel, c->st));
  c->launches++;
  const int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz;
  const size_t cplx = (size_t)nz * ny * (nx / 2 + 1);
  const bool dbl = c->form == FORM_F64;
  if (!c->fft_buf) {
    rc = dev_alloc(c, &c->fft_buf, cplx * (dbl ? 16 : 8), "spectrum buffer");
    if (rc) return rc;
    c->fft_bytes = cplx * (dbl ? 16 : 8);
  }
  if (!c->plan_ok) {
    cufftResult r = cufftPlan3d(&c->plan, nz, ny, nx, dbl ? CUFFT_D2Z : CUFFT_R2C);
    if (r != CUFFT_SUCCESS) {
      set_err("cufftPlan3d failed (%d)", (int)r);
      return BGK_ERR_CUDA;
    }
    c->plan_ok = 1;
    cufftSetStream(c->plan, c->st);
  }
  if (c->nbins_alloc < nbins) {
    if (c->d_bins) {
      cudaFree(c->d_bins);
      c->dev_bytes -= (long long)c->nbins_alloc * 8;
      c->d_bins = nullptr;
    }
    rc = dev_alloc(c, (void**)&c->d_bins, (size_t)nbins * 8, "spectrum bins");
    if (rc) return rc;
    c->nbins_alloc = nbins;
  }
  CK(cudaMemsetAsync(c->d_bins, 0, (size_t)nbins * 8, c->st));
  const size_t n = (size_t)ncell(c);
  const double norm = 1.0 / ((double)n * (double)n);
  for (int d = 0; d < 3; ++d) {
    cufftResult r = dbl ? cufftExecD2Z(c->plan, (double*)c->vel + d * n, (cufftDoubleComplex*)c->fft_buf)
                        : cufftExecR2C(c->plan, (float*)c->vel + d * n, (cufftComplex*)c->fft_buf);
    if (r != CUFFT_SUCCESS) {
      set_err("cufftExec failed (%d)", (int)r);
      return BGK_ERR_CUDA;
    }
    CK(launch_spectrum_bins(c->fft_buf, c->form, nx, ny, nz, nbins, c->d_bins, norm, c->st));
    c->launches++;
  }
  CK(cudaMemcpyAsync(ek, c->d_bins, (size_t)nbins * 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return BGK_OK;
}

// --------------------------------------------------------------- file output
namespace {

constexpr char CKPT_MAGIC[8] = {'B', 'G', 'K', '3', 'D', 'C', 'K', '1'};

struct CkptHeader {
  char magic[8];
  int32_t lx, ly, lz, precision;
  int64_t step;
  double scale, omega;
};

struct FileCloser {
  FILE* f;
  ~FileCloser() {
    if (f) fclose(f);
  }
};

}  // namespace

int bgk_save(bgk_ctx* c, const char* path) {
  int rc = check_init(c);
  if (rc) return rc;
  if (!path) {
    set_err("bgk_save: null path");
    return BGK_ERR_INVALID;
  }
  CK(cudaSetDevice(c->p.device));
  FileCloser fc{fopen(path, "wb")};
  if (!fc.f) {
    set_err("bgk_save: cannot open %s for writing", path);
    return BGK_ERR_INVALID;
  }
  CkptHeader h{};
  std::memcpy(h.magic, CKPT_MAGIC, 8);
  h.lx = c->g.nx; h.ly = c->g.ny; h.lz = c->g.nz; h.precision = c->form;
  h.step = c->step; h.scale = c->scale; h.omega = c->omega;
  if (fwrite(&h, sizeof(h), 1, fc.f) != 1) {
    set_err("bgk_save: write failed on %s", path);
    return BGK_ERR_INVALID;
  }
  const size_t n = (size_t)ncell(c);
  rc = ensure_stage(c, n * 8);
  if (rc) return rc;
  std::vector<char> host(n * c->es);
  for (int q = 0; q < Q; ++q) {
    CK(launch_export(c->A, c->lay, q, c->stage, nullptr, c->scale, c->st));
    c->launches++;
    CK(cudaMemcpyAsync(host.data(), c->stage, n * c->es, cudaMemcpyDeviceToHost, c->st));
    rc = sync_and_check(c);
    if (rc) return rc;
    if (fwrite(host.data(), c->es, n, fc.f) != n) {
      set_err("bgk_save: write failed on %s", path);
      return BGK_ERR_INVALID;
    }
  }
  return BGK_OK;
}

int bgk_load(bgk_ctx* c, const char* path) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!path) {
    set_err("bgk_load: null path");
    return BGK_ERR_INVALID;
  }
  CK(cudaSetDevice(c->p.device));
  FileCloser fc{fopen(path, "rb")};
  if (!fc.f) {
    set_err("bgk_load: cannot open %s", path);
    return BGK_ERR_INVALID;
  }
  CkptHeader h{};
  if (fread(&h, sizeof(h), 1, fc.f) != 1 || std::memcmp(h.magic, CKPT_MAGIC, 8) != 0) {
    set_err("bgk_load: %s is not a checkpoint of this library", path);
    return BGK_ERR_INVALID;
  }
  if (h.lx != c->g.nx || h.ly != c->g.ny || h.lz != c->g.nz || h.precision != c->form) {
    set_err("bgk_load: %s holds a %dx%dx%d box in precision %d, the context is %dx%dx%d in precision %d", path, h.lx,
            h.ly, h.lz, h.precision, c->g.nx, c->g.ny, c->g.nz, c->form);
    return BGK_ERR_INVALID;
  }
  const size_t n = (size_t)ncell(c);
  rc = ensure_stage(c, n * 8);
  if (rc) return rc;
  std::vector<char> host(n * c->es);
  const int lay = init_layout(c);
  for (int q = 0; q < Q; ++q) {
    if (fread(host.data(), c->es, n, fc.f) != n) {
      set_err("bgk_load: %s is truncated", path);
      return BGK_ERR_INVALID;
    }
    CK(cudaMemcpyAsync(c->stage, host.data(), n * c->es, cudaMemcpyHostToDevice, c->st));
    CK(launch_import(c->A, lay, q, c->stage, c->st));
    c->launches++;
    CK(cudaStreamSynchronize(c->st));
  }
  CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st));
  CK(cudaStreamSynchronize(c->st));
  c->lay = lay;
  c->step = h.step;
  c->faith_step[0] = c->faith_step[1] = -1;
  if (c->form == FORM_F16) c->scale = h.scale;
  c->initialized = 1;
  c->faith_step[0] = c->faith_step[1] = -1;
  c->primed = 0;
  return BGK_OK;
}

int bgk_vtk(bgk_ctx* c, int itime, int kind, int index, const char* dir) {
  int rc = check_init(c);
  if (rc) return rc;
  const int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz;
  const int lim = kind == 1 ? nz : kind == 2 ? ny : kind == 3 ? nx : 1;
  if (kind < 0 || kind > 3 || (kind > 0 && (index < 1 || index > lim)) || itime < 0 || itime > 99999999) {
    set_err("bgk_vtk: invalid kind %d / index %d / itime %d", kind, index, itime);
    return BGK_ERR_INVALID;
  }
  CK(cudaSetDevice(c->p.device));
  const long long npts = kind == 1 ? (long long)nx * ny : kind == 2 ? (long long)nx * nz
                       : kind == 3 ? (long long)ny * nz : ncell(c);
  rc = ensure_stage(c, (size_t)npts * 12 > (size_t)ncell(c) * 8 ? (size_t)npts * 12 : (size_t)ncell(c) * 8);
  if (rc) return rc;
  CK(launch_vtk(c->A, c->lay, kind, index - 1, (float*)c->stage, npts, c->scale, c->st));
  c->launches++;
  std::vector<float> v((size_t)npts * 3);
  CK(cudaMemcpyAsync(v.data(), c->stage, (size_t)npts * 12, cudaMemcpyDeviceToHost, c->st));
  rc = sync_and_check(c);
  if (rc) return rc;
  // legacy VTK, as SRC/vtk_xy.binary.F90:58-97 writes it: ASCII header with
  // I10 fields, then big-endian float32 velocity triples; a z-slab writes its
  // own file named by its rank, with its z offset in ORIGIN (offset(3),
  // SRC/vtk_xy.binary.F90:53,65-67), and an xy index local to the slab
  static const char* tag[4] = {"3d", "xy", "xz", "yz"};
  char name[64];
  snprintf(name, sizeof(name), "tec_%s.%05d.%08d.vtk", tag[kind], c->p.coord_z, itime);
  const std::string path = std::string(dir && *dir ? dir : ".") + "/" + name;
  FileCloser fc{fopen(path.c_str(), "wb")};
  if (!fc.f) {
    set_err("bgk_vtk: cannot open %s", path.c_str());
    return BGK_ERR_INVALID;
  }
  const int dims[4][3] = {{nx, ny, nz}, {nx, ny, 1}, {nx, 1, nz}, {1, ny, nz}};
  const int z0 = c->g.z0;
  const int orig[4][3] = {{1, 1, z0 + 1}, {1, 1, z0 + index}, {1, index, z0 + 1}, {index, 1, z0 + 1}};
  fprintf(fc.f, "# vtk DataFile Version 2.0\nCampo\nBINARY\nDATASET STRUCTURED_POINTS\n");
  fprintf(fc.f, "DIMENSIONS %10d %10d %10d\n", dims[kind][0], dims[kind][1], dims[kind][2]);
  fprintf(fc.f, "ORIGIN %10d %10d %10d\n", orig[kind][0], orig[kind][1], orig[kind][2]);
  fprintf(fc.f, "SPACING %10d %10d %10d\n", 1, 1, 1);
  fprintf(fc.f, "POINT_DATA%10lld\n", npts);
  fprintf(fc.f, "VECTORS velocity float \n");
  std::vector<uint32_t> be(v.size());
  for (size_t s = 0; s < v.size(); ++s) {
    uint32_t b;
    std::memcpy(&b, &v[s], 4);
    be[s] = __builtin_bswap32(b);
  }
  if (fwrite(be.data(), 4, be.size(), fc.f) != be.size()) {
    set_err("bgk_vtk: write failed on %s", path.c_str());
    return BGK_ERR_INVALID;
  }
  return BGK_OK;
}

// ------------------------------------------------------------------ adjoint
namespace {

// Hands out lattice-sized device blocks from the context's pool, growing it
// on demand; the blocks stay allocated for later adjoint / tangent calls.
struct AdjBufs {
  bgk_ctx* c;
  size_t next = 0;
  explicit AdjBufs(bgk_ctx* ctx) : c(ctx) {}
  int lattice(Lattice* L, const char* what) {
    if (next == c->lat_pool.size()) {
      void* m = nullptr;
      int rc = dev_alloc(c, &m, (size_t)Q * c->g.qs * c->es, what);
      if (rc) return rc;
      c->lat_pool.push_back(m);
    }
    void* m = c->lat_pool[next++];
    L->form = c->form;
    L->g = c->g;
    for (int q = 0; q < Q; ++q) L->p[q] = (char*)m + (size_t)q * c->g.qs * c->es;
    return BGK_OK;
  }
  int sums(long long n, double** acc, double** tot) {
    if (c->adj_acc_n < n) {
      if (c->adj_acc) {
        cudaFree(c->adj_acc);
        c->dev_bytes -= 2 * c->adj_acc_n * (long long)sizeof(double);
        c->adj_acc = nullptr;
        c->adj_acc_n = 0;
      }
      int rc = dev_alloc(c, (void**)&c->adj_acc, 2 * (size_t)n * sizeof(double), "adjoint sums");
      if (rc) return rc;
      c->adj_acc_n = n;
    }
    if (!c->adj_tot) {
      int rc = dev_alloc(c, (void**)&c->adj_tot, 2 * sizeof(double), "adjoint totals");
      if (rc) return rc;
    }
    *acc = c->adj_acc;
    *tot = c->adj_tot;
    return BGK_OK;
  }
};

// The rebuilt states of a segment of K steps carry the rounding of up to K - 1
// inverted collisions, each of which scales the non-equilibrium part by
// 1 / |1 - omega|, so their relative error grows to about
// K * A * (the form's rounding), A = |1 - omega|^-(K-1). Rebuilding is used
// while A <= 64 and, in FP32 storage (rounding 6e-8), K * A <= 160: a
// rebuilt-state error below about 1e-5, under the 4.5e-5 between the FP32
// and FP64 gradients (FP64: below 1e-12).
bool adj_rebuild_ok(int form, double omega, int K) {
  const double r = std::fabs(1.0 - omega);
  if (!(r > 0.0) || K < 1 || (form != FORM_F64 && form != FORM_F32)) return false;
  const double logA = (K - 1) * std::log(1.0 / r);
  if (logA > std::log(64.0)) return false;
  return form == FORM_F64 || std::log((double)K) + logA <= std::log(160.0);
}

int adj_check(bgk_ctx* c, int nsteps) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (c->form == FORM_F16) {
    set_err("the adjoint and tangent models support the FP64 and FP32 forms");
    return BGK_ERR_INVALID;
  }
  if (c->slab) {
    set_err("the adjoint and tangent models run on a whole box (proc_z = 1)");
    return BGK_ERR_INVALID;
  }
  if (c->p.les_cs > 0.0) {
    set_err("the adjoint and tangent models differentiate the BGK collision (les_cs must be 0)");
    return BGK_ERR_INVALID;
  }
  if (nsteps < 1) {
    set_err("nsteps must be >= 1");
    return BGK_ERR_INVALID;
  }
  return BGK_OK;
}

// Uploads three host arrays of N doubles into velocity buffer `slot`.
int upload3(bgk_ctx* c, int slot, const double* a, const double* b, const double* d, double** out,
            const char* what) {
  const size_t n = (size_t)ncell(c);
  if (!c->vel_pool[slot]) {
    int rc = dev_alloc(c, (void**)&c->vel_pool[slot], 3 * n * sizeof(double), what);
    if (rc) return rc;
  }
  *out = c->vel_pool[slot];
  if (!a) return BGK_OK;  // buffer only (the gradient)
  CK(cudaMemcpyAsync(*out, a, n * 8, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(*out + n, b, n * 8, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(*out + 2 * n, d, n * 8, cudaMemcpyHostToDevice, c->st));
  return BGK_OK;
}

}  // namespace

int bgk_adjoint(bgk_ctx* c, const double* u0, const double* v0, const double* w0, const double* ut, const double* vt,
                const double* wt, int nsteps, int ckpt_every, double* loss, double* grad_u0, double* grad_tau) {
  int rc = adj_check(c, nsteps);
  if (rc) return rc;
  if (!u0 || !v0 || !w0 || !ut || !vt || !wt || !loss || ckpt_every < 1) {
    set_err("bgk_adjoint: invalid argument");
    return BGK_ERR_INVALID;
  }
  CK(cudaSetDevice(c->p.device));
  const int T = nsteps, K = ckpt_every < nsteps ? ckpt_every : nsteps;
  const int nck = (T + K - 1) / K;
  const bool want_grad = grad_u0 || grad_tau;
  // rebuild the states of a segment backwards from the state that ends it
  // when the rounding of K - 1 rebuilt steps grows by at most 64x
  const bool rebuild = want_grad && c->adj_mode == BGK_ADJ_REBUILD && adj_rebuild_ok(c->form, c->omega, K);
  const int nwork = (K - 1 > 2 && !rebuild) ? K - 1 : 2;
  AdjBufs B(c);
  double *du0 = nullptr, *dut = nullptr, *acc = nullptr, *tot = nullptr;
  if ((rc = upload3(c, 0, u0, v0, w0, &du0, "initial velocity"))) return rc;
  if ((rc = upload3(c, 1, ut, vt, wt, &dut, "target velocity"))) return rc;
  const long long nacc = adj_step_blocks(c->g) > DIAG_BLOCKS ? adj_step_blocks(c->g) : DIAG_BLOCKS;
  if ((rc = B.sums(nacc, &acc, &tot))) return rc;
  // segments kept whole in the cache budget (the last ones of the horizon):
  // segment s holds the states t0+1 .. t1-1 between its checkpoint and the next
  const size_t state_bytes = (size_t)Q * c->g.qs * c->es;
  int ncache = 0;
  if (want_grad && K > 1) {
    const size_t per_seg = (size_t)(K - 1) * state_bytes;
    ncache = (int)(c->adj_cache_bytes / per_seg);
    if (ncache > nck) ncache = nck;
  }
  const int s_cache = nck - ncache;  // first cached segment
  std::vector<Lattice> ck(want_grad ? nck : 1), work(want_grad ? nwork : 2), lam(want_grad ? 2 : 1);
  for (auto& L : ck)
    if ((rc = B.lattice(&L, "checkpoint"))) return rc;
  for (auto& L : work)
    if ((rc = B.lattice(&L, "recomputed state"))) return rc;
  for (auto& L : lam)
    if ((rc = B.lattice(&L, "adjoint state"))) return rc;
  std::vector<std::vector<Lattice>> cache(nck);
  for (int s = s_cache; s < nck; ++s) {
    const int t0 = s * K, t1 = t0 + K < T ? t0 + K : T;
    cache[s].resize(t1 - t0 - 1);
    for (auto& L : cache[s])
      if ((rc = B.lattice(&L, "cached forward state"))) return rc;
  }
  // forward: f^0 = equilibrium of u0 at rho = 1, checkpoints every K steps,
  // the states of cached segments into their slots
  const size_t n = (size_t)ncell(c);
  CK(launch_init_velocity(ck[0], LAY_TWO, du0, du0 + n, du0 + 2 * n, 1.0, 0, c->g.nz, 1.0, nullptr, c->st));
  const Lattice* cur = &ck[0];
  int wi = 0;
  for (int t = 0; t < T; ++t) {
    const Lattice* next;
    const int s = t / K, m = t + 1 - s * K;  // f^{t+1} is state m of segment s
    if (want_grad && t + 1 < T && (t + 1) % K == 0) next = &ck[(t + 1) / K];
    else if (want_grad && s >= s_cache && t + 1 < T) next = &cache[s][m - 1];
    else {
      if (cur == &work[wi]) wi ^= 1;
      next = &work[wi];
    }
    CK(launch_step_out_of_place(*cur, *next, c->omega, c->st));
    cur = next;
  }
  CK(cudaMemsetAsync(acc, 0, 2 * DIAG_BLOCKS * sizeof(double), c->st));
  CK(launch_adj_terminal(*cur, dut, lam[0], acc, c->st));
  CK(launch_acc_total(acc, tot, c->st));
  c->launches += T + 3;
  if (want_grad) {
    // backward over the segments, recomputing each from its checkpoint
    CK(cudaMemsetAsync(acc, 0, 2 * nacc * sizeof(double), c->st));
    int li = 0;  // lam[li] holds lam^{t+1}
    for (int s = nck - 1; s >= 0; --s) {
      const int t0 = s * K, t1 = t0 + K < T ? t0 + K : T;
      if (s < s_cache && rebuild) {
        // from f^{t1} (the next checkpoint, or the final state) down to t0:
        // each launch rebuilds g^t into the work lattice it does not read
        const Lattice* post = s == nck - 1 ? cur : &ck[s + 1];
        int gi = post == &work[0] ? 1 : 0;
        for (int t = t1 - 1; t >= t0; --t) {
          const bool first = t == t1 - 1, last = t == t0;
          CK(launch_adj_inv(*post, first, lam[li], lam[li ^ 1], last ? nullptr : &work[gi], c->omega, acc, c->st));
          li ^= 1;
          post = &work[gi];
          gi ^= 1;
        }
        c->launches += t1 - t0;
        continue;
      }
      std::vector<const Lattice*> st(t1 - t0);
      st[0] = &ck[s];
      for (int m = 1; m < t1 - t0; ++m) {
        if (s >= s_cache) {
          st[m] = &cache[s][m - 1];  // kept by the forward pass
        } else {
          CK(launch_step_out_of_place(*st[m - 1], work[m - 1], c->omega, c->st));
          st[m] = &work[m - 1];
          c->launches++;
        }
      }
      for (int t = t1 - 1; t >= t0; --t) {
        CK(launch_adj_step(*st[t - t0], lam[li], lam[li ^ 1], c->omega, acc, c->st));
        li ^= 1;
      }
      c->launches += t1 - t0;
    }
    CK(launch_acc_total_n(acc, adj_step_blocks(c->g), tot + 1, c->st));
    if (grad_u0) {
      double* dg = nullptr;
      if ((rc = upload3(c, 2, nullptr, nullptr, nullptr, &dg, "gradient"))) return rc;
      CK(launch_adj_grad_u0(lam[li], du0, dg, c->st));
      CK(cudaMemcpyAsync(grad_u0, dg, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
      c->launches++;
    }
  }
  double h[2] = {0.0, 0.0};
  CK(cudaMemcpyAsync(h, tot, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  *loss = h[0] / (double)n;
  if (grad_tau) *grad_tau = -c->omega * c->omega * h[1];  // tau = 1/omega
  return BGK_OK;
}

int bgk_adjoint_mode(bgk_ctx* c, int mode) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (mode != BGK_ADJ_RECOMPUTE && mode != BGK_ADJ_REBUILD) {
    set_err("bgk_adjoint_mode: mode must be BGK_ADJ_RECOMPUTE or BGK_ADJ_REBUILD");
    return BGK_ERR_INVALID;
  }
  c->adj_mode = mode;
  return BGK_OK;
}

int bgk_adjoint_rebuilds(int precision, double omega, int ckpt_every) {
  const int form = precision == BGK_FP64 ? FORM_F64 : precision == BGK_FP32DEV ? FORM_F32 : -1;
  return adj_rebuild_ok(form, omega, ckpt_every) ? 1 : 0;
}

int bgk_adjoint_cache(bgk_ctx* c, size_t bytes) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (bytes < c->adj_cache_bytes) {
    // release the pooled lattices; the next call allocates what it needs
    CK(cudaSetDevice(c->p.device));
    CK(cudaStreamSynchronize(c->st));
    const size_t lb = (size_t)Q * c->g.qs * c->es;
    for (void* m : c->lat_pool) cudaFree(m);
    c->dev_bytes -= (long long)(lb * c->lat_pool.size());
    c->lat_pool.clear();
  }
  c->adj_cache_bytes = bytes;
  return BGK_OK;
}

int bgk_tangent(bgk_ctx* c, const double* u0, const double* v0, const double* w0, const double* du0,
                const double* dv0, const double* dw0, double dtau, const double* ut, const double* vt, const double* wt,
                int nsteps, double* loss, double* dloss) {
  int rc = adj_check(c, nsteps);
  if (rc) return rc;
  if (!u0 || !v0 || !w0 || !du0 || !dv0 || !dw0 || !ut || !vt || !wt || !loss || !dloss) {
    set_err("bgk_tangent: invalid argument");
    return BGK_ERR_INVALID;
  }
  CK(cudaSetDevice(c->p.device));
  AdjBufs B(c);
  double *d_u0 = nullptr, *d_du = nullptr, *dut = nullptr, *acc = nullptr, *tot = nullptr;
  if ((rc = upload3(c, 0, u0, v0, w0, &d_u0, "initial velocity"))) return rc;
  if ((rc = upload3(c, 3, du0, dv0, dw0, &d_du, "velocity perturbation"))) return rc;
  if ((rc = upload3(c, 1, ut, vt, wt, &dut, "target velocity"))) return rc;
  if ((rc = B.sums(DIAG_BLOCKS, &acc, &tot))) return rc;
  Lattice f[2], df[2], scratch;
  for (int m = 0; m < 2; ++m) {
    if ((rc = B.lattice(&f[m], "state"))) return rc;
    if ((rc = B.lattice(&df[m], "tangent state"))) return rc;
  }
  if ((rc = B.lattice(&scratch, "scratch"))) return rc;
  const size_t n = (size_t)ncell(c);
  CK(launch_init_velocity(f[0], LAY_TWO, d_u0, d_u0 + n, d_u0 + 2 * n, 1.0, 0, c->g.nz, 1.0, nullptr, c->st));
  CK(launch_tan_init(df[0], d_u0, d_du, c->st));
  const double domega = -c->omega * c->omega * dtau;  // omega = 1/tau
  int cur = 0;
  for (int t = 0; t < nsteps; ++t) {
    CK(launch_tan_step(f[cur], df[cur], f[cur ^ 1], df[cur ^ 1], c->omega, domega, c->st));
    cur ^= 1;
  }
  CK(cudaMemsetAsync(acc, 0, 2 * DIAG_BLOCKS * sizeof(double), c->st));
  CK(launch_adj_terminal(f[cur], dut, scratch, acc, c->st));
  CK(launch_acc_total(acc, tot, c->st));
  CK(cudaMemsetAsync(acc, 0, 2 * DIAG_BLOCKS * sizeof(double), c->st));
  CK(launch_tan_loss(f[cur], df[cur], dut, acc, c->st));
  CK(launch_acc_total(acc, tot + 1, c->st));
  c->launches += nsteps + 6;
  double h[2] = {0.0, 0.0};
  CK(cudaMemcpyAsync(h, tot, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  *loss = h[0] / (double)n;
  *dloss = h[1] / (double)n;
  return BGK_OK;
}

int bgk_get_scale(const bgk_ctx* c, double* s) {
  if (!c || !s) return BGK_ERR_INVALID;
  *s = c->scale;
  return BGK_OK;
}

int bgk_get_omega(const bgk_ctx* c, double* o) {
  if (!c || !o) return BGK_ERR_INVALID;
  *o = c->omega;
  return BGK_OK;
}

int bgk_get_step(const bgk_ctx* c, long long* s) {
  if (!c || !s) return BGK_ERR_INVALID;
  *s = c->step;
  return BGK_OK;
}

int bgk_get_device_bytes(const bgk_ctx* c, long long* b) {
  if (!c || !b) return BGK_ERR_INVALID;
  *b = c->dev_bytes;
  return BGK_OK;
}

int bgk_get_launch_count(const bgk_ctx* c, long long* n) {
  if (!c || !n) return BGK_ERR_INVALID;
  *n = c->launches;
  return BGK_OK;
}

void* bgk_get_stream(const bgk_ctx* c) { return c ? (void*)c->st : nullptr; }

int bgk_synchronize(bgk_ctx* c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  CK(cudaSetDevice(c->p.device));
  return sync_and_check(c);
}

int bgk_record_event(bgk_ctx* c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  CK(cudaSetDevice(c->p.device));
  if (!c->mark) CK(cudaEventCreateWithFlags(&c->mark, cudaEventDisableTiming));
  CK(cudaEventRecord(c->mark, c->st));
  return BGK_OK;
}

int bgk_wait_event(bgk_ctx* c, const bgk_ctx* other) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!other || !other->mark) {
    set_err("bgk_wait_event: the other context has recorded no event (bgk_record_event)");
    return BGK_ERR_STATE;
  }
  CK(cudaSetDevice(c->p.device));
  CK(cudaStreamWaitEvent(c->st, other->mark, 0));
  return BGK_OK;
}

int bgk_shift3(const void* in1, const void* in2, const void* in3, void* out1, void* out2, void* out3, int nx, int ny,
               int nz, int elem_bytes, int reverse, void* stream) {
  if (!in1 || !in2 || !in3 || !out1 || !out2 || !out3 || nx < 1 || ny < 1 || nz < 1 ||
      (elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8)) {
    set_err("bgk_shift3: invalid argument");
    return BGK_ERR_INVALID;
  }
  const void* in[3] = {in1, in2, in3};
  void* out[3] = {out1, out2, out3};
  CK(launch_shift3(in, out, nx, ny, nz, elem_bytes, reverse, (cudaStream_t)stream));
  return BGK_OK;
}

const char* bgk_strerror(int code) {
  switch (code) {
    case BGK_OK: return "ok";
    case BGK_SKIPPED: return "not a diagnostic step";
    case BGK_ERR_INVALID: return "invalid argument";
    case BGK_ERR_CUDA: return "CUDA error";
    case BGK_ERR_NOMEM: return "device memory allocation failed";
    case BGK_ERR_STATE: return "call out of order";
    case BGK_ERR_NONFINITE: return "non-finite density or velocity";
  }
  return "unknown error";
}

const char* bgk_last_error(void) { return g_err; }

const char* bgk_version(void) { return "bgk3d-b200 0.1 (sm_100a)"; }

}  // extern "C"
