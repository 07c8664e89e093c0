/*
 * dda_b200.h -- C ABI of the B200 discrete-dipole-approximation engine.
 *
 * Plain C: device pointers are `void*` / `const void*` to contiguous arrays,
 * sizes are ints, streams are `cudaStream_t` passed as `void*` (NULL = the
 * legacy default stream).  No call synchronises the device; calls that must
 * observe device state (solver termination, cross sections) synchronise only
 * on events of their own internal stream.  Every entry point returns an int
 * status (DDA_OK on success); `dda_last_error()` gives the message of the
 * last failure on the calling thread.
 *
 * Array conventions follow the reference engine (Toastlovesjam/preconDDA):
 *   vectors (polarisation P, incident field E_inc, matvec in/out):
 *       C-order (nx, ny, nz, 3) complex, component index fastest
 *       (Gpbicgstab.py:937, :1172);
 *   inverse polarisability inv_alpha: (nx, ny, nz) complex, 0 outside the
 *       scatterer; the mask is inv_alpha != 0 (ddaforgit.py:1105-1108);
 *   FFT'd interaction tensor ghat: reduced octant (hx, hy, hz) = (Lx/2+1,
 *       Ly/2+1, Lz/2+1) of FFT(-G), components (xx, xy, xz, yy, yz, zz), in
 *       one of two layouts:
 *         DDA_GHAT_REFERENCE  (hx, hy, hz, 6), component fastest -- with
 *             Ln = 2 nn exactly the reference's (nx+1, ny+1, nz+1, 6) array
 *             (ddaforgit.py:1069-1077);
 *         DDA_GHAT_ENGINE     (6, hx, hy, hz), the layout every solver and
 *             matvec entry point reads (coalesced tensor gathers).
 * dtype: DDA_C64 = complex64 (float2), DDA_C128 = complex128 (double2).
 */
#ifndef DDA_B200_H
#define DDA_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define DDA_C64 0
#define DDA_C128 1

/* status codes */
#define DDA_OK 0
#define DDA_ERR_BAD_SHAPE 1
#define DDA_ERR_OOM 2
#define DDA_NOT_CONVERGED 3
#define DDA_ERR_NAN 4
#define DDA_ERR_TIMEOUT 5
#define DDA_ERR_CUDA 6
#define DDA_ERR_ARG 7

/* octant layouts */
#define DDA_GHAT_REFERENCE 0
#define DDA_GHAT_ENGINE 1

/* matvec modes of dda_matvec */
#define DDA_MV_AX 0            /* y = inv_alpha*x - mask*conv(x)          */
#define DDA_MV_RESIDUAL 1      /* y = b - A.x  (b already masked)          */
#define DDA_MV_CONV 2          /* y = conv(x), no mask (near field)        */
#define DDA_MV_CONV_MASKED 3   /* y = mask*conv(x)                         */

typedef struct dda_ctx dda_ctx;
typedef struct dda_op dda_op;

/* One right-hand side of a batched solve.  Instances of one batch share the
 * box (nx,ny,nz), the FFT lengths and the dtype; ghat / inv_alpha may be
 * shared between instances (many incidences of one geometry) or not (many
 * geometries padded into one size bucket). */
typedef struct dda_instance {
  const void* ghat;        /* octant, engine layout, dtype of the solve   */
  const void* inv_alpha;   /* (nx,ny,nz) complex, dtype of the solve      */
  const void* e_inc;       /* (nx,ny,nz,3) complex, dtype of the solve    */
  void* p_out;             /* (nx,ny,nz,3) complex, dtype of the solve    */
} dda_instance;

/* Per-instance result of a solve (reference return tuple, Gpbicgstab.py:1162-1201). */
typedef struct dda_result {
  int iters;               /* i+1 converged, max_iter not converged, -(i+1) NaN / stagnation */
  int status;              /* DDA_OK, DDA_NOT_CONVERGED or DDA_ERR_NAN                       */
  double lowest_rel;       /* lowest recursive residual norm / initial norm                  */
  double first_rel;        /* residual norm after the first iteration / initial norm         */
  double true_relres;      /* ||b - A.P|| / ||b|| where computed (mixed solve), else -1      */
  int outer;               /* refinement sweeps (mixed solve), else 0                        */
  int resets;              /* Krylov restarts taken                                          */
} dda_result;

int dda_version(void);
const char* dda_last_error(void);
/* Number of kernels this library has enqueued in the process so far
 * (instrumentation for benchmarks; no reference counterpart). */
long long dda_kernel_launches(void);

/* Context: device binding, twiddle tables and solver workspaces. */
int dda_ctx_create(int device, dda_ctx** out);
void dda_ctx_destroy(dda_ctx* ctx);
/* Frees cached solver workspaces (they are kept between solves). */
int dda_ctx_trim(dda_ctx* ctx);

/* 1 if L is a usable FFT length for the dtype (even, 2^a 3^b 5^c 7^d,
 * small enough for one shared-memory tile), else 0. */
int dda_fft_length_ok(int L, int dtype);

/* Replaces generate_interaction_row (ddaforgit.py:1046-1080): builds
 * scale * FFT(-G) on the (Lx,Ly,Lz) embedding of the (nx,ny,nz) box, cropped
 * to the octant, in the given layout.  scale = 1 with DDA_GHAT_REFERENCE gives
 * the reference's array.  Writes complex128 to out_c128 and/or complex64 to
 * out_c64 (either may be NULL).  Computed in FP64. */
int dda_green_build(dda_ctx* ctx, int nx, int ny, int nz, int Lx, int Ly, int Lz, double k, double d,
                    double scale, int layout, void* out_c128, void* out_c64, void* stream);

/* Reference-layout octant -> engine layout (same dtype, src != dst). */
int dda_ghat_to_engine(dda_ctx* ctx, int dtype, int hx, int hy, int hz, const void* src, void* dst,
                       void* stream);

/* Operator A for one geometry: references caller-owned ghat (engine layout,
 * multiplied by gscale inside the kernels) and inv_alpha; owns the
 * transform scratch.  Replaces the state prepared by prepare_interaction_matrices
 * (ddaforgit.py:1085-1159) and setup_chunked_values (Gpbicgstab.py:832-876). */
int dda_op_create(dda_ctx* ctx, int dtype, int nx, int ny, int nz, int Lx, int Ly, int Lz, const void* ghat,
                  double gscale, const void* inv_alpha, dda_op** out);
void dda_op_destroy(dda_op* op);

/* Replaces interaction_mult (Gpbicgstab.py:828-830, mode DDA_MV_AX),
 * fft_matvec (Gpbicgstab.py:742-772, DDA_MV_CONV_MASKED) and the product of
 * E_field_solver (ExcitedField.py:129-195, DDA_MV_CONV).  b is read only by
 * DDA_MV_RESIDUAL.  x and y must not alias. */
int dda_matvec(dda_op* op, int mode, const void* x, void* y, const void* b, void* stream);

/* dda_matvec for nb operators / vectors in one launch sequence (every kernel
 * has gridDim.y = nb): operators sharing context, dtype, box, FFT lengths and
 * tensor scale (they may have different ghat / inv_alpha).  Arrays of nb
 * device pointers on the host; b may be NULL unless mode is DDA_MV_RESIDUAL.
 * Uses transform scratch cached in the context per (shape, nb). */
int dda_matvec_batch(dda_op* const* ops, int nb, int mode, const void* const* x, void* const* y,
                     const void* const* b, void* stream);

/* Allocation-free A.x.  No counterpart in the reference.  It serves callers
 * that cannot allocate device memory where they need the product: serving or
 * real-time loops whose latency budget rules out allocator calls (cudaMalloc
 * may synchronise the device and takes unbounded time), and host applications
 * whose device memory belongs to another framework's caching pool, which raw
 * cudaMalloc calls would bypass.  Same product and modes as dda_matvec, with
 * ghat in the engine layout and every array caller-owned; the transform
 * scratch, state block and twiddle tables live in one static __device__
 * array of DDA_NOALLOC_SCRATCH_BYTES that each GPU loading the library keeps
 * until exit.  Problems whose scratch (nx*ny*Lz*3 + nx*Ly*Lz*3 complex) does
 * not fit are rejected with DDA_ERR_BAD_SHAPE (e.g. a 64^3 box with FFT 128^3
 * fits in complex64, not in complex128).  The first call on a device looks up
 * the array's address and writes the twiddle tables with a synchronous copy;
 * it should come before any stream capture.  Later calls only enqueue
 * kernels.  Calls share the array: calls that overlap on the GPU race and
 * must not be issued. */
#define DDA_NOALLOC_SCRATCH_BYTES (64ull << 20)
int dda_matvec_noalloc(int dtype, int nx, int ny, int nz, int Lx, int Ly, int Lz, const void* ghat,
                       double gscale, const void* inv_alpha, int mode, const void* x, void* y, const void* b,
                       void* stream);

/* ---- launch tuning --------------------------------------------------------
 * No counterpart in the reference (its launch shapes are fixed in its CuPy
 * code).  A table, per (dtype, box nx,ny,nz, FFT lengths, batch-width class
 * of nb: 1, 2-3, 4-7, 8-15, 16+), of the matvec launch variant to use, as an
 * autotuner measured it (precondda_b200.batch.LaunchTuner).  Flags:
 *   DDA_TUNE_P3PIPE        the staged persistent x pass (input tiles bulk-
 *                          copied one tile ahead, two CTAs per SM) instead of
 *                          the one-tile-per-CTA kernel, where it is compiled
 *   DDA_TUNE_P3PIPE_1SM    the staged x pass on one CTA per SM
 *   DDA_TUNE_NO_FUSED_ZY   separate z and y forward passes instead of the
 *                          cluster-fused kernel (one-instance launches)
 *   DDA_TUNE_NO_FUSED_INV  separate y and z inverse passes likewise
 *   DDA_TUNE_P3PAIR        the x pass on packed pairs of transforms (FP32x2
 *                          arithmetic, complex64 cubic 64^3 / 128^3 boxes)
 *   DDA_TUNE_YPAIR         the y passes on packed pairs likewise
 *   DDA_TUNE_ZPAIR         the z passes on packed pairs likewise
 *   DDA_TUNE_FUSED         the cluster-fused z/y passes where they are off
 *                          by default (128^3 boxes, launches of any width)
 *   DDA_TUNE_PREFETCH      the x and y passes of cubic boxes prefetch the
 *                          input rows of the tiles one resident wave ahead
 *                          into L2 (bulk prefetches)
 * dda_tuning_set with flags < 0 removes the entry; dda_tuning_get returns
 * DDA_ERR_ARG when there is none.  Entries apply to launches made after
 * the call (a captured iteration graph keeps the variant it was captured
 * with). */
#define DDA_TUNE_P3PIPE 1
#define DDA_TUNE_P3PIPE_1SM 2
#define DDA_TUNE_NO_FUSED_ZY 4
#define DDA_TUNE_NO_FUSED_INV 8
#define DDA_TUNE_P3PAIR 16
#define DDA_TUNE_YPAIR 32
#define DDA_TUNE_ZPAIR 64
#define DDA_TUNE_FUSED 128
#define DDA_TUNE_PREFETCH 256
int dda_tuning_set(int dtype, int nx, int ny, int nz, int Lx, int Ly, int Lz, int nb, int flags);
int dda_tuning_get(int dtype, int nx, int ny, int nz, int Lx, int Ly, int Lz, int nb, int* flags);

/* Replaces solve_gpbicgstab (Gpbicgstab.py:879-1201) with precon=False:
 * solves A.P = E_inc*mask from P0 = 0 with the reference's GPBiCGSTAB
 * recurrence, restarts (ratio), true-residual replacement and return codes.
 * Blocks until the solve ends. */
int dda_gpbicgstab(dda_op* op, const void* e_inc, double target, int max_iter, double ratio, void* p_out,
                   dda_result* res, void* stream);

/* Many right-hand sides / geometries in one batched solve (same box, L and
 * dtype).  Converged instances retire while the others continue. */
int dda_solve_batch(dda_ctx* ctx, int dtype, int nx, int ny, int nz, int Lx, int Ly, int Lz, double gscale,
                    const dda_instance* inst, int nb, double target, int max_iter, double ratio, dda_result* res,
                    void* stream);

/* Mixed precision: complex64 GPBiCGSTAB sweeps (relative target inner_tol
 * for the first; later sweeps aim at 0.8 x what tol still needs) inside an
 * FP64 iterative-refinement loop whose true residual E_inc*mask - A.P is an
 * FP64 matvec; stops when it is <= tol * ||E_inc*mask||.  The sweeps apply
 * the reference's restart rule with max(ratio, 1000) (0: no restarts).
 * inst64 / inst128 describe the same instances in both precisions
 * (inst64[j].p_out and inst64[j].e_inc are scratch the engine may overwrite;
 * inst128[j].p_out receives the FP64 solution). */
int dda_solve_mixed_batch(dda_ctx* ctx, int nx, int ny, int nz, int Lx, int Ly, int Lz, double gscale,
                          const dda_instance* inst64, const dda_instance* inst128, int nb, double tol,
                          double inner_tol, int max_iter, int max_outer, double ratio, dda_result* res,
                          void* stream);

/* ---- preconditioned solves (precon=True) ---------------------------------- */
/* The reference's right-preconditioned GPBiCGSTAB (Gpbicgstab.py:1002-1199,
 * precon=True): A is applied to M p and M s, the residual replacements use
 * A M x and the solution is M x, where
 *   M x = mask * scale * IFFT[ P . FFT(pad x) ]  cropped to the box
 * on the preconditioner's own grid L >= n per axis, P an octant
 * (L/2+1)^3 x 6 read through the interaction octant's mirror rule
 * (fft_matvec3 + optimized_dot_product_reduced_kernel, Gpbicgstab.py:633-668,
 * :36-103; scale = 1/(Lx Ly Lz) for its normalised inverse FFT).  The
 * reference calls preconditioner builders it does not define
 * (ddaforgit.py:1118-1136, pre_preconditioner / circulant_approximation);
 * dda_precond_build is this engine's replacement:
 *   P(q) = [abar I - FFT_L(-c)(q)]^-1,  c(t) = sum_{j = t mod L} w(j) G(j),
 * abar = mean inverse polarizability of the occupied sites, G the lattice
 * Green tensor at offsets j in (-n, n)^3, w(j) the fraction of occupied
 * sites whose neighbour at offset j is occupied (averaged over the 8 axis
 * reflections): the inverse of T. Chan's optimal circulant approximation of
 * the masked operator, folded onto the L-periodic grid (L = n is the
 * cheapest to apply; L = 2n unfolded).  Computed in FP64 from the complex128
 * inverse polarizability; layout DDA_GHAT_REFERENCE (hx,hy,hz,6) or
 * DDA_GHAT_ENGINE (6,hx,hy,hz); either output may be null.  Enqueued on
 * `stream`. */
int dda_precond_build(dda_ctx* ctx, int nx, int ny, int nz, int Lx, int Ly, int Lz, double k, double d,
                      const void* inv_alpha128, int layout, void* out_c128, void* out_c64, void* stream);

/* The preconditioner as an operator (engine-layout octant `phat` on the grid
 * Lx,Ly,Lz >= the box): dda_matvec(pre, DDA_MV_CONV_MASKED, ...) is M x,
 * the reference's fft_matvec3 (Gpbicgstab.py:633-668); inv_alpha supplies
 * the mask.  Destroy with dda_op_destroy. */
int dda_precond_op_create(dda_ctx* ctx, int dtype, int nx, int ny, int nz, int Lx, int Ly, int Lz, const void* phat,
                          double scale, const void* inv_alpha, dda_op** out);

/* dda_gpbicgstab with the preconditioner `pre` (same context, dtype and box
 * as `op`): solve_gpbicgstab(..., precon=True) (Gpbicgstab.py:879-1201). */
int dda_gpbicgstab_pre(dda_op* op, const dda_op* pre, const void* e_inc, double target, int max_iter, double ratio,
                       void* p_out, dda_result* res, void* stream);

/* dda_solve_batch with one preconditioner octant per instance (phat[j],
 * engine layout, dtype of the solve) on the grid Px,Py,Pz, applied with
 * pscale. */
int dda_solve_batch_pre(dda_ctx* ctx, int dtype, int nx, int ny, int nz, int Lx, int Ly, int Lz, double gscale,
                        int Px, int Py, int Pz, double pscale, const void* const* phat, const dda_instance* inst,
                        int nb, double target, int max_iter, double ratio, dda_result* res, void* stream);

/* dda_solve_mixed_batch whose complex64 sweeps are preconditioned
 * (phat64[j]: complex64 engine-layout octants); the FP64 refinement
 * residual is unpreconditioned. */
int dda_solve_mixed_batch_pre(dda_ctx* ctx, int nx, int ny, int nz, int Lx, int Ly, int Lz, double gscale, int Px,
                              int Py, int Pz, double pscale, const void* const* phat64, const dda_instance* inst64,
                              const dda_instance* inst128, int nb, double tol, double inner_tol, int max_iter,
                              int max_outer, double ratio, dda_result* res, void* stream);

/* ---- slot pool: continuous batching ------------------------------------- */
/* A pool of `nslots` solver instances of one box / FFT size that requests
 * enter and leave independently: a request is admitted into a free slot
 * while the other slots keep iterating, all occupied slots advance together
 * through one captured iteration graph, and finished slots are handed back
 * by dda_slots_poll.  Every slot follows solve_gpbicgstab
 * (Gpbicgstab.py:879-1201) exactly as a lone solve would: a slot's result
 * does not depend on what else is in the pool.  The pool runs on its own
 * stream; admit orders itself after `stream`, poll returns with the finished
 * slots' outputs complete. */
#define DDA_PREC_C64 0     /* complex64 GPBiCGSTAB                              */
#define DDA_PREC_C128 1    /* complex128 GPBiCGSTAB                             */
#define DDA_PREC_MIXED 2   /* complex64 sweeps + FP64 refinement (as dda_solve_mixed_batch) */
typedef struct dda_slots dda_slots;

int dda_slots_create(dda_ctx* ctx, int precision, int nx, int ny, int nz, int Lx, int Ly, int Lz, double gscale,
                     int nslots, dda_slots** out);
void dda_slots_destroy(dda_slots* pool);
int dda_slots_capacity(const dda_slots* pool);
/* Index of a free slot, -1 when all are occupied. */
int dda_slots_free_slot(const dda_slots* pool);
/* Admit one request into free slot `slot`.  DDA_PREC_C64 reads `lo`,
 * DDA_PREC_C128 reads `hi`, DDA_PREC_MIXED reads both (lo: complex64 ghat and
 * inv_alpha; hi: complex128 ghat, inv_alpha, e_inc and p_out).  tol is the
 * solver target (the FP64 target for mixed pools); inner_tol, max_outer only
 * matter for mixed pools, whose sweeps follow dda_solve_mixed_batch.  The
 * result lands in p_out when the slot finishes. */
int dda_slots_admit(dda_slots* pool, int slot, const dda_instance* lo, const dda_instance* hi, double tol,
                    double inner_tol, int max_iter, int max_outer, double ratio, void* stream);
/* Preconditioned pools (the precon=True solve of dda_solve_batch_pre for
 * every slot): the preconditioner grid Px,Py,Pz and scale are the pool's;
 * each admitted request brings its own octant `phat` (engine layout,
 * complex64 for DDA_PREC_C64 / DDA_PREC_MIXED, complex128 for DDA_PREC_C128)
 * through dda_slots_admit_pre. */
int dda_slots_create_pre(dda_ctx* ctx, int precision, int nx, int ny, int nz, int Lx, int Ly, int Lz, double gscale,
                         int Px, int Py, int Pz, double pscale, int nslots, dda_slots** out);
int dda_slots_admit_pre(dda_slots* pool, int slot, const dda_instance* lo, const dda_instance* hi, const void* phat,
                        double tol, double inner_tol, int max_iter, int max_outer, double ratio, void* stream);
/* Enqueue `niter` GPBiCGSTAB iterations of every occupied slot. */
int dda_slots_run(dda_slots* pool, int niter);
/* 1 when the pool's stream has finished all enqueued work (dda_slots_poll
 * would not wait), 0 while it is busy, a negative DDA_ERR_* code on error.
 * A host loop over several pools polls the ready ones first, so a pool
 * whose chunk ended is refilled while the others still run. */
int dda_slots_ready(const dda_slots* pool);
/* Wait for the pool's stream, then report the slots that finished since the
 * last poll (finished[0..*nfinished), results in the same order; arrays of
 * capacity length) and free them.  Mixed pools refine here: a finished
 * complex64 sweep is accumulated into the FP64 solution, the FP64 residual is
 * formed, and the slot either finishes or starts another sweep. */
int dda_slots_poll(dda_slots* pool, int* finished, dda_result* results, int* nfinished, int* nrunning);
/* Drop a request (cancellation): the slot becomes free, its output is undefined. */
int dda_slots_release(dda_slots* pool, int slot);

/* ---- lattice setup on the device ---------------------------------------- */
#define DDA_SHAPE_SPHERE 0
#define DDA_SHAPE_ELLIPSOID 1
#define DDA_SHAPE_RECTANGLE 2
#define DDA_SHAPE_CYLINDER 3
#define DDA_SHAPE_PRISM 4

/* Flags of a dda_shape.
 * DDA_SHAPE_WINDOW: the shape marks only sites with win[2a] <= i_a < win[2a+1]
 *   on each axis a -- the per-shape index window of the reference's
 *   mark_shapes (ddaforgit.py:626-649), which bounds its x- and y-axis
 *   cylinders (see below).
 * DDA_SHAPE_GEOMETRIC_AXES: x- and y-axis cylinders take the radial distance
 *   perpendicular to their axis and the absolute axial offset.  Without it a
 *   cylinder follows the reference's Numba cylinder (ddaforgit.py:477-509):
 *   the radial distance is always taken in the (x, y) plane, and for the x
 *   and y axes the height test compares the signed z offset with height/2. */
#define DDA_SHAPE_WINDOW 1
#define DDA_SHAPE_GEOMETRIC_AXES 2

/* One shape of a voxelisation, in the length unit of d.  p[]: sphere r;
 * ellipsoid semi-axes (a,b,c); rectangle edge lengths (x,y,z); cylinder
 * (radius, height); prism (circumradius, height).  axis (0,1,2 = x,y,z) for
 * cylinder / prism, sides for prism.  rot: ellipsoid body->lab rotation,
 * row-major (identity for the reference's axis-aligned ellipsoid).
 * inv_alpha: value written at member sites.  flags / win: see above (win in
 * the voxelised box's site indices). */
typedef struct dda_shape {
  int type;
  int axis;
  int sides;
  int flags;
  double center[3];
  double p[4];
  double rot[9];
  double inv_alpha[2];
  int win[6];
  int reserved[2];
} dda_shape;

/* Replaces mark_shapes / create_alpha_and_n_arrays (ddaforgit.py:615-830)
 * for a given box: voxelises shapes into inv_alpha (nx,ny,nz) at voxel
 * centres origin + (i+0.5) d; a site takes the value of the last shape
 * containing it, 0 if none.  Membership tests as the reference's
 * (ddaforgit.py:439-572), evaluated on the GPU; shapes is a host array. */
int dda_voxelize(dda_ctx* ctx, int dtype, const dda_shape* shapes, int nshape, int nx, int ny, int nz, double d,
                 const double* origin3, void* inv_alpha_out, void* stream);

/* Plane wave E = e exp(i k.r), r = (i,j,k) d, as the reference builds E_inc
 * (ddaforgit.py:1626-1632); pol6 = (Re ex, Im ex, Re ey, Im ey, Re ez, Im ez). */
int dda_incident_field(dda_ctx* ctx, int dtype, int nx, int ny, int nz, double d, const double* k3,
                       const double* pol6, void* e_out, void* stream);

/* Extinction, absorption and scattering cross sections (Draine & Flatau
 * 1994, not present in the reference) reduced in FP64:
 *   out[0] = C_ext = 4 pi k/|E0|^2 sum Im(E_inc* . P)
 *   out[1] = C_abs = 4 pi k/|E0|^2 sum [Im(P . conj(inv_alpha) P*) - 2/3 k^3 |P|^2]
 *   out[2] = C_sca = C_ext - C_abs
 * All three arrays have the given dtype; sites with inv_alpha == 0 are skipped. */
int dda_cross_sections(dda_ctx* ctx, int dtype, long long nsite, const void* p, const void* e_inc,
                       const void* inv_alpha, double k, double e0, double* out3, void* stream);

/* Far-field scattering amplitude (not in the reference; Draine 1988):
 *   F(n) = k^2 sum_j [P_j - n (n . P_j)] exp(-i k n . r_j),  r_j = (i,j,k) d
 * for ndir (1..65535) directions dirs3 (host, 3 doubles each, normalised here); out6
 * (host, 6 doubles per direction) = (Re F_x, Im F_x, Re F_y, Im F_y, Re F_z,
 * Im F_z).  dC_sca/dOmega = |F|^2 / |E0|^2; F at the incidence direction
 * gives C_ext = 4 pi / k Im(E0* . F) / |E0|^2.  Sums in FP64, phases
 * from FP64 sincos; blocks until the result is on the host. */
int dda_far_field(dda_ctx* ctx, int dtype, int nx, int ny, int nz, double d, double k, const void* p, int ndir,
                  const double* dirs3, double* out6, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* DDA_B200_H */
