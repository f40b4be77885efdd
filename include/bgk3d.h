/*
 * bgk3d.h - C-ABI of the B200 implementation of the BGK3D_HIT time-step hot
 * path (D3Q19 BGK, triply periodic box, one GPU).
 *
 * The entry points mirror the reference's Fortran call sequence
 * (SRC/bgk3d_HIT.F90:74-92 set-up, :127-146 time loop):
 *
 *     input + setup_MPI + hencol + alloca  ->  bgk_create
 *     init                                 ->  bgk_init_tgv / bgk_init_velocity
 *     do itime = 1, itfin
 *        boundaries(itime)                 ->  bgk_boundaries   (no-op: the
 *                                              periodic wrap is inside the kernel)
 *        col_MC(itime)                     ->  bgk_col_mc
 *        diagnostic(itime, icheck, ...)    ->  bgk_diagnostic
 *     end do
 *     finalize                             ->  bgk_destroy
 *
 * Conventions
 *  - Every function returns BGK_OK (0) on success, a negative BGK_ERR_* code
 *    on error, and never exits the process (the reference stops instead,
 *    e.g. SRC/input.F90:66-82). bgk_last_error() gives a message.
 *  - Host arrays are Fortran order (i fastest) without ghost layers; a
 *    population array is q-major: element (q, i, j, k), q = 0..18 for the
 *    reference's a01..a19, sits at q*lx*ly*lz + i + lx*(j + ly*k).
 *  - Populations are deviations f_q - w_q (the reference's default storage,
 *    cte1 = 1 in SRC/col_MC.F90:86-90), in the stored precision; the FP16
 *    form stores scale*(f_q - w_q).
 *  - A context is not thread-safe. Its work runs in order on one CUDA stream
 *    owned by the context; calls that return host data synchronise it.
 *  - The library allocates the device memory it uses in bgk_create and on
 *    first use of a feature that needs more (diagnostics, spectrum, host
 *    transfers, the adjoint and its state cache), keeps it for later calls
 *    and frees it in bgk_destroy. bgk_diagnostics_noalloc allocates nothing.
 */
#ifndef BGK3D_H
#define BGK3D_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BGK_OK 0
#define BGK_SKIPPED 1          /* bgk_diagnostic: not a diagnostic step */
#define BGK_ERR_INVALID (-1)   /* bad argument or parameter */
#define BGK_ERR_CUDA (-2)      /* CUDA runtime error */
#define BGK_ERR_NOMEM (-3)     /* device allocation failed */
#define BGK_ERR_STATE (-4)     /* call out of order (e.g. step before init) */
#define BGK_ERR_NONFINITE (-5) /* diagnostics found non-finite moments */

/* Storage / arithmetic forms (SRC/precision.F90:19-38 has DOUBLE_P and the
   single-precision default; the FP16 form has no working reference
   counterpart, SRC/precision.F90:40-43). */
#define BGK_FP64 0    /* double storage, double arithmetic */
#define BGK_FP32DEV 1 /* float storage of f - w, float arithmetic */
#define BGK_FP16DEV 2 /* binary16 storage of scale*(f - w), float arithmetic */

/* Update schemes. */
#define BGK_TWO_LATTICE 0 /* pull stream-collide a -> b and swap, SRC/col_MC.F90:98-421 */
#define BGK_AA 1          /* in-place AA pattern, one lattice (no reference counterpart) */

/* Modes. */
#define BGK_CORRECTED 0 /* TGV init in double with rho = 1; diagno sums ztot */
#define BGK_FAITHFUL 1  /* TGV init with single-precision coordinates, pi and the
                           pressure-consistent crho (SRC/init.F90:42,84-95);
                           diagno keeps ztot = ytot + zj (SRC/diagno.F90:110);
                           on a whole two-lattice box, dissipation pulls the
                           reference's stale ghost cells (it runs after the
                           pointer swap: after step t >= 2 the ghosts hold the
                           state of step t - 2, after step 1 zero deviations);
                           sums stay compensated FP64 in both modes */

typedef struct bgk_ctx bgk_ctx;

/* Run parameters: the reference's namelist &parameters (SRC/input.F90:41-47)
   restricted to one box, plus the build-time choices of the reference
   (precision, scheme) as run-time values. */
typedef struct {
  int lx, ly, lz;      /* box size (SRC/input.F90:61-63; one rank: l = lx ...) */
  double svisc;        /* kinematic viscosity nu; omega = 2/(6 nu + 1), SRC/hencol.F90:31 */
  double u0;           /* reference velocity (TGV amplitude, dissipation.dat normalisation) */
  int precision;       /* BGK_FP64 / BGK_FP32DEV / BGK_FP16DEV */
  int scheme;          /* BGK_TWO_LATTICE / BGK_AA */
  int icheck;          /* diagnostic interval (SRC/diagnostic.F90:37) */
  int mode;            /* BGK_CORRECTED / BGK_FAITHFUL */
  double fp16_scale;   /* FP16 form: scale (power of two); 0 = chosen at init */
  int device;          /* CUDA device ordinal */
  int use_omega;       /* 1: use `omega` below instead of the svisc formula */
  double omega;        /* collision frequency override (e.g. 0 = pure streaming) */
  int extras;          /* 1: bgk_diagnostic also computes enstrophy */
  int kernel;          /* stream-collide kernel: 0 automatic (FP16: 4 where the box
                          fits, FP32: 2 where it fits, else 1; the BGK odd step of the
                          AA scheme on 8 (FP16) / 4 (FP32) cells per thread where the
                          box fits that), 1 one cell per thread,
                          2 two cells per thread (FP32 both schemes, FP16 two-lattice),
                          4 four cells per thread (FP16), 8 row pipeline with TMA bulk
                          copies into shared memory (rows up to about 5 KB); boxes a
                          kernel does not fit use 1. All give identical results. */
  double les_cs;       /* Smagorinsky constant cteS (SRC/input.F90:47, SRC/storage.F90:87).
                          > 0 enables the LES collision of SRC/col_MC.F90:221-309 (the
                          block the reference compiles under -DLES and then stops in):
                          per cell Ptotal = |Pi_neq|, Ts = 1/(2 omega) +
                          sqrt(18 cteS^2 Ptotal + (1/omega)^2)/2, relaxation with 1/Ts.
                          0 (default) = plain BGK. The LES collision runs on the one
                          cell per thread kernels, in FP32 on the two (the AA odd
                          step: four) and in FP16 on the four cells per thread
                          kernels where the box fits (FP16 kernel 2 and kernel 8
                          fall back);
                          bgk_adjoint and bgk_tangent reject it. */
  int proc_z;          /* number of z-slabs the box is split into (the reference's
                          proc_z, SRC/input.F90:41; proc_x = proc_y = 1). 1 (default):
                          one whole periodic box. > 1: this context holds slab
                          coord_z, lz/proc_z planes starting at global plane
                          coord_z*lz/proc_z (lz is the global height and must be a
                          multiple of proc_z, as SRC/input.F90:66-82 requires); see
                          "z-slabs" below. */
  int coord_z;         /* this slab's index, 0..proc_z-1 (the rank's z coordinate in
                          the reference's MPI_Cart topology, SRC/setup_MPI.F90:112-131) */
} bgk_params;

/* Diagnostics of one step, in FP64. */
typedef struct {
  int itime;
  /* diagno.dat columns, SRC/diagno.F90:117-137 (means over the box of the
     local, un-pulled populations) */
  double rho_mean, ux_mean, uy_mean, uz_mean, ke_mean;
  /* dissipation.dat columns, SRC/dissipation.F90:261-269 (pulled populations):
     t = itime*dt, tke_norm = sum(0.5|u|^2)/(l m n u0^2), diss = sum(2 svisc Ptotal) */
  double t, tke_norm, diss;
  double tke;          /* sum(0.5|u|^2) over the pulled populations, unnormalised */
  double enstrophy;    /* mean 0.5|curl u|^2 (central differences), no reference counterpart */
  double eps_strain;   /* mean 2 nu S:S, S = -3 omega Pi_neq/(2 rho), no reference counterpart */
  long long nonfinite; /* cells with non-finite local rho or u */
} bgk_diag;

/* Fills defaults: 64^3, svisc 0.01, u0 0.05, FP64, two-lattice, icheck 10,
   corrected mode, device 0, extras on. */
int bgk_params_default(bgk_params* p);

/* = input + setup_MPI + hencol + alloca (SRC/bgk3d_HIT.F90:74-89). Validates
   the parameters, selects the device, allocates the lattice(s). */
int bgk_create(const bgk_params* p, bgk_ctx** out);

/* = finalize's teardown (SRC/finalize.F90): frees everything. NULL is ok. */
int bgk_destroy(bgk_ctx* ctx);

/* = init (SRC/init.F90:23-163): Taylor-Green vortex with amplitude u0. */
int bgk_init_tgv(bgk_ctx* ctx);

/* Equilibrium initial condition from a host velocity field (three arrays of
   lx*ly*lz doubles, Fortran order) at uniform density rho; the per-cell
   arithmetic of SRC/init.F90:97-137 with crho = rho. Used for decaying HIT. */
int bgk_init_velocity(bgk_ctx* ctx, const double* u, const double* v, const double* w, double rho);

/* Same as bgk_init_velocity with the three velocity arrays in device memory
   of the context's device (lx*ly*lz doubles each, Fortran order), read in
   place: no host copy and no staging buffer. For fields made on the GPU
   (large HIT boxes) or held by a device runtime. Arrays of another device or
   host memory are rejected with BGK_ERR_INVALID. No reference counterpart
   (SRC/init.F90 builds its field on the host). */
int bgk_init_velocity_device(bgk_ctx* ctx, const double* u, const double* v, const double* w, double rho);

/* = boundaries(itime) (SRC/boundaries.F90:23-107, default STEP3 variant
   SRC/bcond.comm.step3.F90:29-316). The single periodic box needs no halo
   exchange: every kernel wraps its indices. Kept so that the call sequence is
   unchanged; validates the context and returns BGK_OK. */
int bgk_boundaries(bgk_ctx* ctx, int itime);

/* = col_MC(itime) (SRC/col_MC.F90:34-444): one fused pull-stream + BGK
   collide step over the box, including the a <-> b swap (two-lattice) or the
   layout flip (AA). Asynchronous. */
int bgk_col_mc(bgk_ctx* ctx, int itime);

/* Runs nsteps consecutive bgk_boundaries + bgk_col_mc steps. Asynchronous. */
int bgk_run(bgk_ctx* ctx, int nsteps);

/* = diagnostic(itime, icheck, ...) (SRC/diagnostic.F90:25-75): when
   mod(itime, icheck) == 0 computes diagno + dissipation (+ enstrophy when
   params.extras) into *out and returns BGK_OK (or BGK_ERR_NONFINITE when
   out->nonfinite > 0); otherwise returns BGK_SKIPPED and leaves *out alone.
   Synchronous. */
int bgk_diagnostic(bgk_ctx* ctx, int itime, bgk_diag* out);

/* = diagno(itime) (SRC/diagno.F90:28-154): out[5] = {mean rho, mean ux,
   mean uy, mean uz, mean 0.5|u|^2}. Ungated. */
int bgk_diagno(bgk_ctx* ctx, int itime, double* out5);

/* = dissipation(itime) (SRC/dissipation.F90:176-280): out[4] = {itime*dt,
   tke_norm, diss, tke}. Ungated. */
int bgk_dissipation(bgk_ctx* ctx, int itime, double* out4);

/* Current populations in the reference's meaning (post-collision a_q of
   SRC/col_MC.F90 after the swap), stored type (double / float / binary16
   bits), q-major Fortran order. */
int bgk_get_populations(bgk_ctx* ctx, void* host19);
int bgk_put_populations(bgk_ctx* ctx, const void* host19);
/* Same as bgk_get_populations, decoded to double deviations f_q - w_q. */
int bgk_get_deviations(bgk_ctx* ctx, double* host19);
/* Local velocity u = j/rho of every cell (as in SRC/diagno.F90:100-104). */
int bgk_get_velocity(bgk_ctx* ctx, double* u, double* v, double* w);

/* Shell-averaged kinetic-energy spectrum of the local velocity field:
   E[k] = sum over wavevectors with round(|k|) == k of 0.5|u_hat|^2 / N^2,
   k = 0..nbins-1 (cuFFT). No reference counterpart. */
int bgk_spectrum(bgk_ctx* ctx, int nbins, double* ek);

/* Checkpoint / restart of the populations (the reference reads itsave and
   irestart, SRC/input.F90:41-42, but never saves or restarts). bgk_save
   writes a small header (box, precision, step, scale, omega) and the 19
   populations in the reference's meaning and order; bgk_load restores them
   into a context of the same box and precision (either scheme) and sets its
   step counter (and the FP16 scale). Synchronous. */
int bgk_save(bgk_ctx* ctx, const char* path);
int bgk_load(bgk_ctx* ctx, const char* path);

/* VTK output as the reference's vtk_*_bin subroutines write it
   (SRC/vtk_xy.binary.F90:58-97, vtk_xz / vtk_yz / vtk_3d): legacy
   STRUCTURED_POINTS, BINARY, big-endian float32 velocity j/rho, file
   tec_<kind>.00000.<itime, 8 digits>.vtk in `dir` (NULL: current directory).
   kind 1: xy plane at z = index, 2: xz at y = index, 3: yz at x = index
   (1-based, as the reference's k0, j0, i0), 0: the whole box (index ignored).
   Synchronous. */
int bgk_vtk(bgk_ctx* ctx, int itime, int kind, int index, const char* dir);

/* Discrete adjoint of the time loop (no reference counterpart). From the
   initial velocity (u0, v0, w0) (equilibrium at rho = 1, as bgk_init_velocity),
   runs nsteps stream-collide steps with the context's omega, and computes
   loss = 0.5 mean |u(T) - u_tgt|^2 over the box (u: local velocity of the final
   populations), grad_u0 = dloss/d(u0, v0, w0) (3 blocks of lx*ly*lz doubles)
   and grad_tau = dloss/dtau, tau = 1/omega. The backward pass recomputes the
   forward from checkpoints stored every ckpt_every steps (about sqrt(nsteps)
   keeps memory at (nsteps/ckpt_every + ckpt_every + 2) lattices). grad_u0 and
   grad_tau may be NULL (with both NULL only the loss is computed). FP64 and
   FP32 forms; works in device buffers of its own, which stay allocated in the
   context for later calls (bgk_destroy frees them), and leaves the context's
   populations unchanged. Synchronous. */
int bgk_adjoint(bgk_ctx* ctx, const double* u0, const double* v0, const double* w0, const double* u_tgt,
                const double* v_tgt, const double* w_tgt, int nsteps, int ckpt_every, double* loss,
                double* grad_u0, double* grad_tau);

/* Device memory (bytes, default 0) that bgk_adjoint may spend on keeping the
   forward states between checkpoints, so that the backward pass need not
   recompute them: whole segments of ckpt_every - 1 states are kept, the last
   segments of the horizon first, as many as fit. With the whole horizon kept
   (ckpt_every - 1 states per segment) the recomputation disappears; results
   are identical either way. The states stay allocated in the context like the
   other adjoint buffers; a smaller budget frees them. */
int bgk_adjoint_cache(bgk_ctx* ctx, size_t bytes);

/* How bgk_adjoint's backward pass obtains the forward states between
   checkpoints (no reference counterpart).
   BGK_ADJ_RECOMPUTE (default): runs the forward again from each checkpoint
   and keeps the segment's states; the gradient is the exact discrete adjoint
   of the stored trajectory.
   BGK_ADJ_REBUILD: rebuilds them backwards from the state that ends each
   segment, inside the adjoint step: the BGK collision keeps rho and j, so the
   post-collision populations x of a cell give the pre-collision ones
   g = (x - omega e(x)) / (1 - omega). No recomputation and no segment states
   (2 work lattices instead of ckpt_every - 1): one backward step moves
   4 x 19 populations per cell against 19 + 19 (recomputation) + 3 x 19
   (adjoint step). The rebuilt states equal the forward's up to rounding,
   which grows by up to 1/|1 - omega| per rebuilt step: with
   A = |1 - omega|^-(ckpt_every - 1), the mode applies where A <= 64 and, in
   the FP32 form, ckpt_every * A <= 160 (bgk_adjoint_rebuilds), and
   bgk_adjoint recomputes otherwise. Cached segments (bgk_adjoint_cache) use
   their kept states in either mode. */
#define BGK_ADJ_RECOMPUTE 0
#define BGK_ADJ_REBUILD 1
int bgk_adjoint_mode(bgk_ctx* ctx, int mode);
/* 1 when BGK_ADJ_REBUILD applies to the form `precision` (BGK_FP64 or
   BGK_FP32DEV), omega and ckpt_every, else 0. */
int bgk_adjoint_rebuilds(int precision, double omega, int ckpt_every);

/* Tangent-linear run (forward-mode derivative) of the same loss: dloss is the
   derivative of loss along the perturbation (du0, dv0, dw0) of the initial
   velocity and dtau of tau. Used to check bgk_adjoint:
   dloss == <grad_u0, du> + grad_tau * dtau. FP64 and FP32 forms. */
int bgk_tangent(bgk_ctx* ctx, const double* u0, const double* v0, const double* w0, const double* du0,
                const double* dv0, const double* dw0, double dtau, const double* u_tgt, const double* v_tgt,
                const double* w_tgt, int nsteps, double* loss, double* dloss);

/* Scale of the FP16 form (1.0 for the other forms). */
int bgk_get_scale(const bgk_ctx* ctx, double* scale);
/* omega in use (SRC/hencol.F90:31 in the form's arithmetic, or the override). */
int bgk_get_omega(const bgk_ctx* ctx, double* omega);
/* Number of steps taken since the last init. */
int bgk_get_step(const bgk_ctx* ctx, long long* step);
/* Device bytes allocated by the context. */
int bgk_get_device_bytes(const bgk_ctx* ctx, long long* bytes);
/* Number of kernel launches issued by the context so far. */
int bgk_get_launch_count(const bgk_ctx* ctx, long long* count);
/* The context's CUDA stream (a cudaStream_t), for event timing by callers. */
void* bgk_get_stream(const bgk_ctx* ctx);
/* Waits for all work of the context. */
int bgk_synchronize(bgk_ctx* ctx);
/* Device-side ordering between contexts of one process (on one or several
   devices), without a host wait: bgk_record_event marks the work queued so
   far on ctx's stream; bgk_wait_event makes ctx's later work wait for the
   work `other` had queued at its last bgk_record_event. */
int bgk_record_event(bgk_ctx* ctx);
int bgk_wait_event(bgk_ctx* ctx, const bgk_ctx* other);

/* z-slabs (proc_z > 1): the halo exchange of bcond_comm_step3
   (SRC/bcond.comm.step3.F90:77-297, five populations per z face) without
   messages. Each slab owns a ghost buffer: two step parities x two faces x
   five populations x one lx*ly plane (padded rows). The step kernel reads its
   own ghost planes and stores its boundary planes' crossing populations
   directly into the neighbours' ghost buffers for the next step - device
   pointers that may live on another GPU (peer stores over NVLink / NVSwitch).
   Contract for the caller (one process per GPU, or several slabs in one
   process):
     1. bgk_halo_buffer / bgk_halo_ipc_handle: publish each slab's buffer;
     2. bgk_halo_connect(ctx, below, above): give each slab the buffers of
        slabs coord_z-1 and coord_z+1 (mod proc_z) as device pointers usable
        from its device (same process: the pointers themselves; another
        process: bgk_halo_ipc_open);
     3. after every initial condition, bgk_put_populations or bgk_load:
        bgk_halo_prime on every slab;
     4. between consecutive bgk_col_mc / bgk_halo_prime / diagnostic calls of
        different slabs, every slab's previous call must have completed on the
        device before any slab's next call starts (a barrier: a stream-ordered
        collective such as a one-element NCCL all-reduce on the contexts'
        streams; in one process, bgk_record_event on every slab and then
        bgk_wait_event of each slab on its two neighbours; or
        bgk_synchronize on every slab plus a host barrier).
   bgk_col_mc then advances one slab by one step (bgk_run accepts nsteps <= 1),
   the diagnostics return this slab's contribution to the global means (sums
   divided by the global cell count: the global value is the sum over the
   slabs), and bgk_vtk writes the slab's file with its rank number and z
   offset as the reference's per-rank writers do. z-slabs run the
   two-lattice scheme in corrected mode; FP16 needs an explicit fp16_scale
   (the same on every slab); enstrophy, bgk_spectrum, bgk_adjoint and
   bgk_tangent are not available on a slab. */
/* This slab's ghost buffer (device pointer and size in bytes). */
int bgk_halo_buffer(const bgk_ctx* ctx, void** dptr, size_t* bytes);
/* cudaIpcGetMemHandle of the ghost buffer into handle[64]. */
int bgk_halo_ipc_handle(const bgk_ctx* ctx, void* handle64);
/* Maps another process's ghost buffer (handle from bgk_halo_ipc_handle) into
   this context's device; the mapping is released by bgk_destroy. */
int bgk_halo_ipc_open(bgk_ctx* ctx, const void* handle64, void** dptr);
/* Sets the ghost buffers of the slab below (coord_z - 1) and above
   (coord_z + 1), periodic in coord_z; enables peer access when they are on
   another device of this process. */
int bgk_halo_connect(bgk_ctx* ctx, void* below, void* above);
/* Stores this slab's boundary planes into the neighbours' ghost buffers for
   the current step (after an initial condition, upload or restart). */
int bgk_halo_prime(bgk_ctx* ctx);

/* Duration in microseconds of the last step's edge-plane kernel of a z-slab
   (the boundary planes that read the ghost planes and store into the
   neighbours'), timed on the device with events while the interior kernel
   runs beside it on the context's second stream. Waits for that step.
   BGK_ERR_STATE before the slab's first step. No reference counterpart (the
   reference's timers, SRC/finalize.F90:58-63, time its MPI exchange). */
int bgk_slab_edge_time(bgk_ctx* ctx, double* us);

/* Streaming-only calibrator, the single-box equivalent of do_somethingGPU
   (SRC/do_somethingGPU.F90:37-100) without the MPI barrier: out1(i,j,k) =
   in1(i-1,j,k), out2 = in2(i,j-1,k), out3 = in3(i,j,k-1) with periodic wrap
   (reverse = 1: +1 shifts, the REVERSE validation mode). Device pointers of
   dense Fortran-order nx*ny*nz arrays of elem_bytes = 2, 4 or 8; stream may
   be NULL (default stream). Asynchronous. */
int bgk_shift3(const void* in1, const void* in2, const void* in3, void* out1, void* out2, void* out3, int nx, int ny,
               int nz, int elem_bytes, int reverse, void* stream);

/* Diagnostics without any allocation, for callers that cannot allocate device
   memory once their time loop runs (a driver whose device arrays all belong
   to another runtime, such as an OpenACC data region, or an application that
   gives all device memory to its own pool; cudaMalloc can fail on a full
   device and synchronises it). No counterpart in the reference.
   Computes the bgk_diagnostic fields except enstrophy (left 0) over caller-
   owned device populations in the reference's meaning: pops19[q] is the
   device base of population q, cell (i,j,k) at i + pitch_x*(j + ly*k), stored
   as `precision` (FP16: scale fp16_scale). Only the rows may be padded
   (pitch_x >= lx); planes follow each other every pitch_x*ly cells, so a
   driver that keeps the reference's ghosted (0:l+1, 0:m+1, 0:n+1) arrays
   passes a copy of their interior, not the ghosted arrays themselves. svisc and omega enter the
   dissipation and strain sums, u0 and itime the dissipation.dat columns, mode
   the diagno ztot convention (without a history of earlier states, its
   dissipation pulls are periodic in both modes). Runs on the calling thread's
   current device and
   on `stream` (NULL: default stream), then synchronises that stream.
   Scratch: one file-scope device array of 94,808 bytes per GPU (held until the
   process exits), whatever the box size; boxes are limited to
   pitch_x*ly*lz < 2^31 cells per population and larger ones are rejected with
   BGK_ERR_INVALID. The array keeps the last call's contents; every slot is
   rewritten before it is read, but calls that overlap on the GPU (concurrent
   streams, threads) race on it. Every call looks up the array's device
   address in the calling thread's current context (cudaGetSymbolAddress);
   the first call in a context also loads the library's kernels there, so
   make that first call before any stream capture. Calls no cudaMalloc or
   cudaFree. */
int bgk_diagnostics_noalloc(const void* const* pops19, int lx, int ly, int lz, int pitch_x, int precision,
                            double svisc, double omega, double u0, double fp16_scale, int mode, int itime,
                            bgk_diag* out, void* stream);

/* Test hook for the failure path of the row-pipelined kernel (params.kernel
   = 8): during the next bgk_col_mc its first CTA waits on a barrier that
   nothing arms; the bounded wait runs out, the step is abandoned and the next
   synchronising call returns BGK_ERR_CUDA. The context stays usable after a
   new bgk_init_* or bgk_put_populations. Faults nothing. */
int bgk_debug_stall_next_step(bgk_ctx* ctx);

const char* bgk_strerror(int code);
/* Message of the last error on this thread. */
const char* bgk_last_error(void);
/* Library version string. */
const char* bgk_version(void);

#ifdef __cplusplus
}
#endif
#endif /* BGK3D_H */
