// Host-side launchers of the library's kernels (internal interface between
// the C-ABI layer and the kernels; not exported).
#pragma once
#include <cuda_runtime.h>
#include "lattice.cuh"

namespace bgk {

enum Form { FORM_F64 = 0, FORM_F32 = 1, FORM_F16 = 2 };
// How the reference's a_q(x) (post-collision, not yet streamed) is stored:
//   LAY_TWO : two-lattice, slot q at x
//   LAY_AAE : AA pattern after an even step / after init, slot opp(q) at x
//   LAY_AAN : AA pattern after an odd step, slot q at x + c_q
enum Layout { LAY_TWO = 0, LAY_AAE = 1, LAY_AAN = 2 };

struct Lattice {
  int form;
  Geo g;
  void* p[Q];          // population base pointers
  int* err = nullptr;  // device flag set by a pipelined kernel whose wait ran out
  int stall = 0;       // test hook: the next pipelined launch waits on a barrier nothing arms
};

// Ghost-plane pointers of a z-slab for one step (see Halo in lattice.cuh):
// in_lo / in_hi this slab's planes read this step, up / dn the neighbours'
// planes written for the next step.
struct SlabLinks {
  void* in_lo[NZF];
  void* in_hi[NZF];
  void* up[NZF];
  void* dn[NZF];
};

// Modes of the row-pipelined kernel (rows.cu).
enum RowMode { ROW_TWO = 0, ROW_AA_EVEN = 1, ROW_AA_ODD = 2 };

// Number of accumulated diagnostic quantities (see kernels.cu).
constexpr int ND = 10;
constexpr int DIAG_BLOCKS = 148 * 4;
constexpr int DIAG_THREADS = 256;

// Collision constants of one launch for a form.
StepK make_stepk(int form, double omega, double scale, double les_cs = 0.0);

// Two-lattice fused pull-stream + collide: src -> dst (pops 1..18), pop 19 in
// place in src. variant: 0 automatic, 1 one cell per thread, 2 / 4 cells per
// thread for the FP16 form, 8 row pipeline with TMA bulk copies (each falls
// back to 1 where the box does not fit it).
cudaError_t launch_two_lattice(const Lattice& src, const Lattice& dst, double omega, double scale, double les_cs,
                               int variant, cudaStream_t st);
// One step src -> dst with all 19 populations written to dst (pop 19 too);
// FP64 and FP32 forms (used by the adjoint's recomputation).
cudaError_t launch_step_out_of_place(const Lattice& src, const Lattice& dst, double omega, cudaStream_t st);

// ------------------------------------------------------------- adjoint
// Terminal adjoint and loss: lam = dL/df for L = 0.5 mean|u(f) - u_tgt|^2;
// the loss is accumulated into acc (one compensated pair per block).
cudaError_t launch_adj_terminal(const Lattice& f, const double* ut, const Lattice& lam, double* acc, cudaStream_t st);
// lam_out = (d step / d f_t)^T lam_in, with f_t the state before the step;
// accumulates -sum(lam_in . (g - e)) = dL/domega of this step into acc, one
// compensated pair per block of the launch (adj_step_blocks pairs).
long long adj_step_blocks(const Geo& g);
cudaError_t launch_acc_total_n(const double* acc, long long n, double* total, cudaStream_t st);
cudaError_t launch_adj_step(const Lattice& ft, const Lattice& lam_in, const Lattice& lam_out, double omega,
                            double* acc, cudaStream_t st);
// The same adjoint step on a state rebuilt from the one after it: post is the
// state after the step, read unshifted (first: a stored forward state) or,
// when first is false, the g that the previous launch rebuilt (gathered from
// x + c_q); writes lam_out and, when gout is not null, the rebuilt
// pre-collision g for the next launch. Same launch shape and acc pairs as
// launch_adj_step.
cudaError_t launch_adj_inv(const Lattice& post, bool first, const Lattice& lam_in, const Lattice& lam_out,
                           const Lattice* gout, double omega, double* acc, cudaStream_t st);
// dL/du0 (3 dense arrays) from lam at t = 0 and the initial velocity u0.
cudaError_t launch_adj_grad_u0(const Lattice& lam0, const double* u0, double* grad, cudaStream_t st);
// Tangent-linear model: perturbation of the initial state from du0 ...
cudaError_t launch_tan_init(const Lattice& df, const double* u0, const double* du0, cudaStream_t st);
// ... one step of (f, df) -> (f', df') with omega perturbed by domega ...
cudaError_t launch_tan_step(const Lattice& f, const Lattice& df, const Lattice& f2, const Lattice& df2, double omega,
                            double domega, cudaStream_t st);
// ... and dL = mean (u - u_tgt).du at the final state into acc.
cudaError_t launch_tan_loss(const Lattice& f, const Lattice& df, const double* ut, double* acc, cudaStream_t st);
// Sums the per-block pairs of acc (DIAG_BLOCKS pairs) into *total.
cudaError_t launch_acc_total(const double* acc, double* total, cudaStream_t st);

// AA pattern: even (local read, reversed local write) or odd (pull from
// neighbours' opposite slots, push to neighbours). variant as above (1 or 8).
cudaError_t launch_aa(const Lattice& a, int odd, double omega, double scale, double les_cs, int variant,
                      cudaStream_t st);
// Row-pipelined kernel; *launched = false when the box does not fit it.
cudaError_t launch_rows(const Lattice& src, const Lattice& dst, int mode, const StepK& K, cudaStream_t st,
                        bool* launched);

// Initial conditions (write layout `lay`, which must be LAY_TWO or LAY_AAE).
// mx != nullptr: only measure max |f - w| into *mx (bits of a float), no store.
cudaError_t launch_init_tgv(const Lattice& a, int lay, double u0, int faithful, double scale, unsigned int* mx,
                            cudaStream_t st);
cudaError_t launch_init_velocity(const Lattice& a, int lay, const double* u, const double* v, const double* w,
                                 double rho, int k0, int nk, double scale, unsigned int* mx, cudaStream_t st);

// Population q in reference semantics, dense Fortran order.
cudaError_t launch_export(const Lattice& a, int lay, int q, void* dense_stored, double* dense_dev, double scale,
                          cudaStream_t st);
cudaError_t launch_import(const Lattice& a, int lay, int q, const void* dense_stored, cudaStream_t st);

// Faithful-mode ghosts: the six boundary planes (x = 0, nx-1; y = 0, ny-1;
// z = 0, nz-1) of every population of a two-lattice state, stored type,
// population-major; faith_planes_elems is the size of one snapshot.
long long faith_planes_elems(const Geo& g);
cudaError_t launch_faith_snapshot(const Lattice& a, void* out, cudaStream_t st);

// Diagnostics: per-block partial sums (Neumaier pairs) of ND quantities.
// vel (optional, 3*N values of the arithmetic type) receives the local velocity.
// halo: the ghost planes of a z-slab (in_lo / in_hi), nullptr for a whole box.
// faith (two-lattice only): pulls that leave the box read the periodic image
// from this boundary-plane snapshot instead of the current state; with
// faith_zero they read a zero deviation (ghosts never written).
cudaError_t launch_diag(const Lattice& a, int lay, double svisc, double omega, double scale, double* partials,
                        void* vel, cudaStream_t st, const SlabLinks* halo = nullptr, const void* faith = nullptr,
                        bool faith_zero = false);

// z-slab two-lattice step (src -> dst, pop 19 in place) reading the ghost
// planes links.in_* and storing the outgoing boundary populations into
// links.up / links.dn: the boundary planes on st, the interior planes on
// st_interior (the caller orders the two streams); and the fill of
// links.up / links.dn from the current state alone.
cudaError_t launch_slab(const Lattice& src, const Lattice& dst, const SlabLinks& links, double omega, double scale,
                        double les_cs, cudaStream_t st, cudaStream_t st_interior);
cudaError_t launch_halo_prime(const Lattice& a, const SlabLinks& links, cudaStream_t st);
cudaError_t launch_enstrophy(const Lattice& a, const void* vel, double* partials, cudaStream_t st);
// Sums DIAG_BLOCKS partials into ND totals (fixed order, compensated).
cudaError_t launch_finalize(const double* partials, double* totals, cudaStream_t st);
// Faithful-mode helper: zj of the last cell (i=l, j=m, k=n) into *out.
cudaError_t launch_last_zj(const Lattice& a, int lay, double scale, double* out, cudaStream_t st);

// Shell binning of one transformed velocity component (nz x ny x (nx/2+1)
// complex values of the arithmetic type): bins[round(|k|)] += w*0.5|u_hat|^2*norm.
cudaError_t launch_spectrum_bins(const void* fft_out, int form, int nx, int ny, int nz, int nbins, double* bins,
                                 double norm, cudaStream_t st);

// Velocity float triples of a VTK slice (kind 1 xy at z = index, 2 xz at
// y = index, 3 yz at x = index; 0-based) or of the box (kind 0), in file order.
cudaError_t launch_vtk(const Lattice& a, int lay, int kind, int index, float* out, long long npts, double scale,
                       cudaStream_t st);

// Streaming-only calibrator (shift of three scalar fields by one cell).
cudaError_t launch_shift3(const void* const in[3], void* const out[3], int nx, int ny, int nz, int elem_bytes,
                          int reverse, cudaStream_t st);

// Sets the message returned by bgk_last_error() on this thread.
void set_last_error(const char* msg);

}  // namespace bgk
