/*
 * fame_b200.h -- C ABI of the B200-native band-structure path of FAME-Isotropic-GPU.
 *
 * One shared library (fame-isotropic-gpu_b200/libfame_b200.so) exports these
 * symbols with C linkage.  Signatures use plain pointers and sizes only.  Every
 * entry point returns an int status (FAME_OK = 0) and never exits or asserts;
 * fame_last_error() returns a message for the calling thread's last failure.
 *
 * Conventions shared with the reference (relative to its project root):
 *   - grid (Nx, Ny, Nz) is the reference's adjusted grid (FAME_Preprocessing/
 *     FAME_Parameter_Generator.cpp:106-112), N = Nx*Ny*Nz;
 *   - edge permittivities B are 3N doubles, x-, y-, z-edge blocks, index
 *     i + Nx*(j + Ny*k) (FAME_Main/FAME_Matrix_B_Isotropic.cu:4-74);
 *   - wave vectors are Cartesian without the 2*pi factor, in the computational
 *     frame (FAME_Main/FAME_Matrix_Lambdas.cu:43-45);
 *   - eigenvectors E are 3N complex128 per band, stored as (re, im) pairs, band
 *     major, scaled like the reference's Eigen_Restoration_Isotropic
 *     (FAME_Main/FAME_Fast_Algorithms_Isotropic.cu:90-125).
 */
#ifndef FAME_B200_H
#define FAME_B200_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
  FAME_OK = 0,
  FAME_ERR_BAD_INPUT = 1,
  FAME_ERR_NO_CONVERGENCE = 2,
  FAME_ERR_WATCHDOG = 3,
  FAME_ERR_CUDA = 4,
  FAME_ERR_NO_DEVICE = 5,
  FAME_ERR_UNSUPPORTED = 6,
  FAME_ERR_IO = 7
};

/* precision modes */
enum { FAME_FP64 = 0, FAME_MIXED = 1 };

/* operators for fame_apply (device pointers, one k-point) */
enum {
  FAME_OP_QR = 0,   /* y(3N) = Q_r x(2Nd)     FAME_Matrix_Vector_Production_Qr.cu:8-78  */
  FAME_OP_QRS = 1,  /* y(2Nd) = Q_r^* x(3N)   FAME_Matrix_Vector_Production_Qrs.cu:7-58 */
  FAME_OP_QBQ = 2,  /* y(2Nd) = Q_r^* B^-1 Q_r x   …Isotropic_QBQ.cu:8-67              */
  FAME_OP_PR = 3,   /* y(3N) = P_r x(2Nd)     FAME_Matrix_Vector_Production_Pr.cu:11-104 */
  FAME_OP_PRS = 4,  /* y(2Nd) = P_r^* x(3N)   FAME_Matrix_Vector_Production_Prs.cu:9-58 */
  FAME_OP_INVAR = 5 /* y(2Nd) = A_r^-1 x      …Isotropic_invAr.cu:8-48 (CG inside)    */
};

typedef struct fame_ctx fame_ctx;

/* Lattice of the computation.  Replaces the grid / lattice part of the reference's
 * PAR struct (include/FAME_Internal_Common.h:64-99,179-187). */
typedef struct {
  int grid[3];              /* Nx, Ny, Nz */
  double mesh_len[3];       /* hx, hy, hz (Par.mesh.mesh_len) */
  double lattice_vec_a[9];  /* computational-frame a1, a2, a3 (Par.lattice.lattice_vec_a) */
  int simple;               /* 1: simple_cubic / primitive_orthorhombic / primitive_tetragonal */
  int m[4];                 /* m1..m4 boundary shifts (General lattices) */
  double t1[3];             /* boundary translation t1 (General lattices) */
} fame_lattice;

/* Solver parameters (the reference's ES and LS, include/FAME_Internal_Common.h:157-167). */
typedef struct {
  int nwant;        /* ES.nwant */
  int nstep;        /* ES.nstep (<= 64) */
  int es_maxit;     /* ES.maxit: maximum Lanczos restarts */
  double es_tol;    /* ES.tol: |beta_m z_m,i| < tol */
  int ls_maxit;     /* LS.maxit */
  double ls_tol;    /* LS.tol: absolute ||r|| of the inner solve */
  int precision;    /* FAME_FP64 or FAME_MIXED */
  int batch;        /* k-points per launch (0 = automatic: what 60% of free device memory holds, <= 64) */
  int use_graph;    /* 1 = run each batch as one CUDA graph (default), 0 = host-driven loop */
  double inner_tol; /* FAME_MIXED: relative tolerance of each FP32 inner solve (0 = 2e-6) */
  int inner_maxit;  /* FAME_MIXED: products per FP32 inner solve (0 = 200) */
  int want_vectors; /* 1 = compute and return the eigenvectors E */
} fame_solver_params;

/* Per k-point counters (the reference's PROFILE, include/FAME_Internal_Common.h:205-211,
 * plus the mixed-precision breakdown). */
typedef struct {
  int ls_iter;      /* Profile.ls_iter: CG products (reference counting, CG.cu:36-77) */
  int es_iter;      /* Profile.es_iter: A_r^-1 applications */
  int restarts;     /* Lanczos restarts */
  int status;       /* FAME_OK / FAME_ERR_NO_CONVERGENCE for this k */
  int Nd;           /* N or N-1 (Gamma point) */
  int refine;       /* FAME_MIXED: FP64 refinement steps (each one FP64 Q_r^* B^-1 Q_r); else 0 */
  int detail;       /* why status is FAME_ERR_NO_CONVERGENCE, FAME_KSTATUS_* bits (0 when FAME_OK) */
} fame_kcounters;

/* fame_kcounters.detail bits.  The reference only prints these cases
 * (FAME_Main/CG.cu:81-84, FAME_Main/Lanczos_Isotropic.cu:84-85). */
#define FAME_KSTATUS_QL 1      /* the tridiagonal eigensolve did not converge */
#define FAME_KSTATUS_LANCZOS 2 /* Lanczos stopped at es_maxit restarts unconverged */
#define FAME_KSTATUS_CG 4      /* an A_r^-1 solve stopped above ls_tol: ls_maxit products (FP64) or
                                  the refinement cap (FAME_MIXED) */

/* Create a context on `device` for one lattice/grid.  Allocates nothing per k yet.
 * FAME_ERR_BAD_INPUT before any allocation: a grid dimension below 2, a mesh length
 * that is not finite and positive, a lattice vector or shift that is not finite.
 * FAME_ERR_UNSUPPORTED: an axis needing more than 10 FFT passes, or an FP64 plane
 * (mid x fast) beyond one CTA's shared memory. */
int fame_ctx_create(int device, const fame_lattice* lat, fame_ctx** out);
void fame_ctx_destroy(fame_ctx* ctx);

/* Edge permittivities B (3N doubles, host).  Replaces FAME_Matrix_B_Isotropic's
 * output (FAME_Main/FAME_Matrix_B_Isotropic.cu:4-74). */
int fame_set_eps(fame_ctx* ctx, const double* B_eps);

/* B from the reference's material index map Binout (3 * material_num * N ints,
 * FAME_Preprocessing/FAME_Material_Locate_Index.cpp:101-113) with the same
 * last-material-wins rule as FAME_Matrix_B_Isotropic.cu:41-61. */
int fame_set_material(fame_ctx* ctx, const int* binout, int material_num, const double* eps_in,
                      double eps_out);

/* Solve nk k-points (k_xyz: 3*nk doubles).  Outputs (host, caller owned):
 *   freq_out   nk*nwant   omega = sqrt(1/theta) per band (FAME_Fast_Algorithms_Isotropic.cu
 *                         + Lanczos_Isotropic.cu:88, Gamma patch :61-79);
 *   relres_out nk*nwant   ||C^H C E - w^2 B E|| / (w^2 ||B E||) evaluated in FP64, or NULL;
 *   relerr_out nk*nwant   |w^2 - rho| / rho with rho the FP64 Rayleigh quotient of the
 *                         band's own Ritz vector (the library's FP64 check of each
 *                         eigenvalue; not a comparison with a separate FP64 solve), or NULL;
 *   resabs_out nk*nwant   ||C^H C E - w^2 B E|| for E scaled as the reference restores it
 *                         (FAME_Fast_Algorithms_Isotropic.cu:119-121), the quantity its
 *                         Check_Residual tests against 1e-10 (FAME_Main_Code.cu:383-421),
 *                         or NULL (non-NULL adds one Q_r apply per band);
 *   evec_out   nk*nwant*3N complex128 (params->want_vectors), or NULL: with
 *              want_vectors set and evec_out NULL the eigenvectors stay on the device
 *              for fame_adjoint_vjp (all nk k-points must fit one batch);
 *   counters   nk entries, or NULL.
 * FAME_ERR_BAD_INPUT, before any device work: NULL k_xyz, params or freq_out, nk < 1,
 * a wave vector with a NaN or infinite component, no permittivity set, parameters
 * outside 1 <= nwant < nstep <= 64, es_maxit >= 0, ls_maxit >= 1, tolerances > 0, or
 * a precision other than FAME_FP64 / FAME_MIXED.
 * Replaces FAME_Fast_Algorithms_Driver (FAME_Main/FAME_Main_Code.cu:142-171) over
 * the k-loop of FAME_Main_Code (:79-133). */
int fame_solve_kpoints(fame_ctx* ctx, const double* k_xyz, int nk, const fame_solver_params* params,
                       double* freq_out, double* relres_out, double* relerr_out, double* resabs_out,
                       double* evec_out, fame_kcounters* counters);

/* Apply one operator at one k-point on device buffers (complex, interleaved):
 * in/out are device pointers of length given in the FAME_OP_* comments.
 * precision: FAME_FP64 (complex128 buffers) or FAME_MIXED (complex64 buffers, not
 * for FAME_OP_INVAR).  For FAME_OP_INVAR ls_tol / ls_maxit come from `params`.
 * Returns Nd through *Nd_out when not NULL. */
int fame_apply(fame_ctx* ctx, int op, const double* k_xyz, const void* in, void* out, int precision,
               const fame_solver_params* params, int* Nd_out);

/* Hellmann-Feynman adjoint for the isotropic problem C^H C E = w^2 B E:
 * dw_i/dB_e = -(w_i/2) |E_i,e|^2 / (E_i^H B E_i) for every edge e, summed over the
 * three edges of each voxel (B_x = B_y = B_z = eps per voxel).  evec is the
 * device or host array returned by fame_solve_kpoints for one k (nwant*3N complex128),
 * `host` tells which.  grad_out: nwant*N doubles (host). */
int fame_adjoint(fame_ctx* ctx, const double* freq, const double* evec, int nwant, int host,
                 double* grad_out);

/* Edge permittivities B (3N doubles) in DEVICE memory of the context's device, for
 * callers that keep the permittivity on the GPU (inverse design).  Entries that are
 * not finite and positive are rejected with FAME_ERR_BAD_INPUT before anything is
 * written.  Same effect as fame_set_eps otherwise. */
int fame_set_eps_device(fame_ctx* ctx, const double* B_eps_device);

/* Vector-Jacobian product of the band frequencies for one k-point of the last
 * fame_solve_kpoints call that kept its eigenvectors on the device (want_vectors set,
 * evec_out NULL, all k-points in one batch): grad_device[v] = sum_i grad_w[i]
 * dw_i/deps_v for one permittivity per voxel (the Hellmann-Feynman form of
 * fame_adjoint), written to N doubles of device memory.  freq and grad_w are the
 * nwant frequencies of that k-point and their weights (host).  Bands whose relative
 * gap is at most rel_gap form degenerate groups: the derivative of a single band of a
 * group is not defined, so unequal weights inside a group are FAME_ERR_BAD_INPUT;
 * equal weights give the derivative of the group's sum.  No counterpart in the
 * reference, which has no adjoint. */
int fame_adjoint_vjp(fame_ctx* ctx, int kidx, const double* freq, const double* grad_w, int nwant,
                     double rel_gap, double* grad_device);

/* The context's CUDA stream (a cudaStream_t), so callers can time work on it with
 * CUDA events.  All device work of the context runs on this stream. */
void* fame_ctx_stream(fame_ctx* ctx);

/* Number of kernels of this library launched on the device so far (counted on the
 * device by every kernel's first thread, graph-launched kernels included). */
int fame_launch_count(fame_ctx* ctx, unsigned long long* count_out);

/* Bound on the trips of every device loop of later solves on this context: the CG,
 * refinement, inner FP32 and Lanczos restart loops each stop after at most
 * `max_trips` trips (0 restores the defaults: ls_maxit + 2, 42, inner_maxit + 2 and
 * es_maxit + 2, which only a fault reaches).  A loop that reaches its bound ends the
 * solve with FAME_ERR_WATCHDOG instead of running on.  No counterpart in the
 * reference, whose loops are host-driven. */
int fame_set_loop_cap(fame_ctx* ctx, int max_trips);

/* Execution options of a context, used by later solves and operator applies (they
 * change how the kernels run; the results agree to rounding):
 *   "prefetch"         1: each CTA of the mixed-precision CG's stage kernels issues L2
 *                      prefetches of the operands of the CTA one wave later; 0 (default): none.
 *   "radix_order"      0..3: radix order of the FFT plans of runtime-geometry grids
 *                      (every grid but the compile-time 96^3 one); 0 is the default.
 *   "plane_threads32", "plane_threads64": threads of a runtime-geometry plane CTA in the
 *                      FP32 / FP64 kernels, a multiple of 32 in 64..512, or 0 for the
 *                      built-in rule.
 *   "self_prefetch"    1 (default): the CG plane stages prefetch their own operands into L2
 *                      at the CTA's start; 0: off.
 *   "static_planes"    1 (default): the plane stages of the FCC 64x55x52, BCC 48x45x39 and
 *                      hexagonal 128x107x92 grids run compile-time FFT plans (fixed CTA
 *                      sizes; the plane-thread options do not apply to them); 0: runtime plans.
 *   "lanes"            1..8 (default 2): fame_solve_kpoints with an automatic batch
 *                      (params.batch 0), at least 4 k-points per lane and eigenvectors not
 *                      kept on the device splits the k-points into this many contiguous
 *                      blocks, each solved concurrently by a lane context (own stream, own
 *                      host thread, this context's permittivity and options); 1: one batch.
 *                      Lowering the value frees the lane contexts (and their device memory)
 *                      it no longer needs; a call whose lane contexts cannot be created
 *                      runs as one batch.
 * Read-only (fame_get_option): "static96", "general", "grid_x", "grid_y", "grid_z",
 * "level" (the FFT pass level the grid needs).  fame_tune picks the first four by timing.
 * Unknown names or values are FAME_ERR_BAD_INPUT.  No counterpart in the reference. */
int fame_set_option(fame_ctx* ctx, const char* name, int value);
int fame_get_option(fame_ctx* ctx, const char* name, int* value);

/* FFT plan autotuner: picks the execution options above ("radix_order",
 * "plane_threads32"/"plane_threads64", "prefetch") for this context's grid by timing
 * candidates on `batch` copies of wave vector k (CUDA events, L2 flushed before each
 * repetition): one FP32 CG iteration for FAME_MIXED, one FP64 Q_r^* B^-1 Q_r apply for
 * FAME_FP64.  The winner is applied to the context.  cache_file (or NULL): a text
 * file of "key | plan" lines, key = grid, lattice family, precision and batch; a
 * cached plan is applied without timing, a new one is appended.  plan_out (or NULL)
 * receives the plan as text.  Replaces the fixed cuFFT plans of the reference
 * (FAME_Main/FAME_Create_cublas.cu:16-25). */
int fame_tune(fame_ctx* ctx, const double* k, int precision, int batch, const char* cache_file, char* plan_out,
              int plan_len);

/* Operator benchmark: `reps` applications of Q_r^* B^-1 Q_r at wave vector k in
 * FP64 (precision FAME_FP64) or FP32 (FAME_MIXED) to a batch of `nbatch` vectors
 * (1..64, the k-point repeated in every slot, as the solver batches k-points), each
 * preceded by an L2 flush (a 256 MiB device write) outside the timed span; CUDA
 * events on the context stream.  stage_ms_out[3] (optional) receives the mean
 * device time of the plane inverse stage, the pencil stage and the plane forward
 * stage over the whole batch; ms_out the mean of their sum. */
int fame_bench_qbq(fame_ctx* ctx, const double* k, int precision, int reps, int nbatch, double* ms_out,
                   double* stage_ms_out);

/* CG-iteration benchmark: `reps` iterations of the mixed-precision solve's FP32 CG
 * (the three kernels of one iteration: search direction and solution update with
 * the 2 -> 3 mix and the inverse plane transforms; slow-axis transforms with <p, Ap>;
 * forward plane transforms with the 3 -> 2 unmix, r -= a Ap and ||r||^2) on `nbatch`
 * k-points (1..64, the k-point repeated), from a fixed pseudo-random residual, each
 * iteration preceded by an L2 flush outside the timed span.  stage_ms_out[3]
 * (optional) receives the mean time of the three kernels over the batch, ms_out
 * their sum.  The CG iteration of FAME_Main/CG.cu:36-77 on QBQ. */
int fame_bench_cg(fame_ctx* ctx, const double* k, int reps, int nbatch, double* ms_out, double* stage_ms_out);

/* Grid size N and maximum reduced size 2N of the context, for buffer sizing. */
int fame_ctx_sizes(const fame_ctx* ctx, long long* N_out);

/* Geometry of the material map (the reference's PAR fields, include/FAME_Internal_Common.h:64-99,
 * 124-131): grid = Par.mesh.grid_nums, mesh_len = Par.mesh.mesh_len, lattice_vec_a and Omega
 * = Par.lattice.lattice_vec_a / Omega (column major), permutation = Par.lattice.Permutation. */
typedef struct {
  int grid[3];
  double mesh_len[3];
  double lattice_vec_a[9];
  double Omega[9];
  int permutation[3];
} fame_locate_geometry;

/* Shapes of each material (Par.material, include/FAME_Internal_Common.h:93-110): material m
 * owns sphere_num[m] spheres and cylinder_num[m] cylinders, listed material by material;
 * centres are fractional coordinates of the original lattice (3 doubles each). */
typedef struct {
  int material_num;
  const int* sphere_num;
  const double* sphere_centers;
  const double* sphere_radius;
  const int* cylinder_num;
  const double* cylinder_top_centers;
  const double* cylinder_bot_centers;
  const double* cylinder_radius;
} fame_material_shapes;

/* The material index map Binout (host, 3 * material_num * N ints: x-, y-, z-edge blocks, each
 * material_num blocks of N, 1 where the edge point lies in that material, the first material
 * that contains it) computed on `device`, bit-exact with the reference's CPU
 * FAME_Material_Locate_Index (FAME_Preprocessing/FAME_Material_Locate_Index.cpp:6-113,
 * FAME_Material_Handle.cpp:4-87).  Feed it to fame_set_material. */
int fame_material_locate(int device, const fame_locate_geometry* geo, const fame_material_shapes* mat,
                         int* binout);

/* Bytes of the fixed device scratch array behind fame_qbq_static. */
#define FAME_QBQ_STATIC_SCRATCH_BYTES (4u << 20)

/* Q_r^* B^-1 Q_r in FP64 at one k-point with no device allocation and no context.
 * No counterpart in the reference (it allocates its work arrays in FAME_Main_Code);
 * this is for callers that own all device memory through their own pool or must
 * not call cudaMalloc/cudaFree (which synchronise the device).
 *   lat     host lattice description (same as fame_ctx_create)
 *   k_xyz   host wave vector (3 doubles)
 *   inv_b   device, 3N doubles: 1/eps per edge (x, y, z components, spatial layout)
 *   x, y    device, 2*Nd complex128 each (Nd = N, or N-1 at the Gamma point)
 *   stream  a cudaStream_t (NULL: the legacy default stream); the call only
 *           enqueues work and returns without synchronising.
 * Scratch is one static device array of FAME_QBQ_STATIC_SCRATCH_BYTES per device
 * (48 bytes per grid point plus tables: grids up to about 85,000 points); larger
 * grids return FAME_ERR_UNSUPPORTED.  Every call shares that array and leaves its
 * contents behind (nothing in it has to start at zero); calls that can overlap in
 * time race on it, so the caller serialises them.  The first call on a device
 * looks up the array's address and keeps it for the life of the process; make it
 * before any stream capture.  The address belongs to the device's primary context:
 * calls from a non-primary (driver-API) context, or after cudaDeviceReset, are not
 * supported. */
int fame_qbq_static(const fame_lattice* lat, const double* k_xyz, const double* inv_b, const void* x, void* y,
                    void* stream);

/* Eigenvector text files in the reference's format: replaces FAME_Save_Eigenvector
 * (FAME_Tools/FAME_Save_Eigenvector.cpp:7-45, called from FAME_Main/FAME_Main_Code.cu:127).
 * For band b of wave vector kidx it writes <dir>/Data_EV_<kk>_<bb>.txt (kk = kidx + 1,
 * bb = b + 1, at least two digits) holding the line "Ele_field_mtx{kk}(:, bb) = [",
 * then one "(% e) + (% e * 1i)" line per entry and "];", byte for byte what the
 * reference's writer produces.  The lines are formatted on `nthreads` host threads
 * (0: all hardware threads) and written in order.
 *   dir     directory (NULL or "": the working directory)
 *   evec    host, nwant x n3 complex128 (band-major, n3 = 3N): one wave vector's
 *           eigenvectors as fame_solve_kpoints returns them
 * fame_writer_start does the same on a background thread and returns at once; the
 * caller keeps `evec` unchanged until fame_writer_finish(writer) has returned, which
 * joins the thread, frees the writer and returns the write's status. */
typedef struct fame_writer fame_writer;
int fame_write_eigenvectors(const char* dir, const double* evec, int nwant, long long n3, int kidx, int nthreads);
int fame_writer_start(const char* dir, const double* evec, int nwant, long long n3, int kidx, int nthreads,
                      fame_writer** writer_out);
int fame_writer_finish(fame_writer* writer);

const char* fame_last_error(void);
const char* fame_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FAME_B200_H */
