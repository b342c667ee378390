/*
 * dns_b200.h -- C ABI of libdnsb200.so, a B200 (sm_100a) implementation of
 * the v-omega Fourier-Chebyshev DNS time step of Riveryh/gpu-spectral-
 * channel-DNS (rotating plane Couette / channel flow; AB2 nonlinear, CN
 * linear, 3/2-padded dealiasing, Chebyshev collocation walls).
 *
 * Plain pointers and sizes only.  Every call returns a dns_status; on error
 * dns_last_error() gives a message (per thread).  Device pointers are
 * CUDA device addresses on the context's device; all work is ordered on
 * the context's stream (dns_get_stream) and is asynchronous unless stated.
 *
 * Layouts follow the reference (include/data.h:189-334):
 *   spectral "ZXY"  complex double [ky][kx][k], ky < Nz, kx < Kx = Nx/2+1,
 *                   pencil pitch `tpitch` bytes (reference tPitch);
 *   physical "XYZ"  double [z][y][x], z < Py = mz/2+1 wall-normal points,
 *                   y < Pz = my spanwise, x < Px = mx, row pitch `pitch`
 *                   bytes (reference pitch); the same buffer holds complex
 *                   rows of mx/2+1 entries before the streamwise transform.
 * Axis names are the reference's: x streamwise, y spanwise, z wall-normal;
 * reference "w" is the wall-normal velocity, "omega_z" the wall-normal
 * vorticity; the solver state is (w, omega_z) = (v, omega_y) in standard
 * notation, with pencil (0,0) holding the mean u0 / w0 profiles.
 */
#ifndef DNS_B200_H
#define DNS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DNS_B200_ABI_VERSION 2

typedef struct dns_ctx dns_ctx;

typedef enum dns_status {
  DNS_OK = 0,
  DNS_ERR_ARG = 1,         /* bad argument / unsupported size */
  DNS_ERR_CUDA = 2,        /* CUDA runtime error */
  DNS_ERR_STATE = 3,       /* call out of order (e.g. step before state) */
  DNS_ERR_TIMEOUT = 4,     /* a device wait ran past its iteration limit */
  DNS_ERR_SINGULAR = 5,    /* an operator matrix had a zero pivot */
  DNS_ERR_IO = 6,          /* file could not be read / parsed */
  DNS_ERR_NONFINITE = 7    /* state contains NaN or Inf */
} dns_status;

/* direction and padding enums of the reference
 * (include/transpose.cuh:9-11, include/transform.cuh:13) */
enum { DNS_FORWARD = 0, DNS_BACKWARD = 1 };
enum { DNS_PADDING = 0, DNS_NO_PADDING = 1 };
/* arithmetic of the transform / nonlinear path */
enum { DNS_PREC_FP64 = 0, DNS_PREC_MIXED = 1 };
/* where a host-facing buffer lives */
enum { DNS_HOST = 0, DNS_DEVICE = 1 };

/* Numerical parameters: the first three records of parameter.txt
 * (include/parameters.h:4-13, source/operation.cpp:123-127) plus the base
 * flow U(y) = U0 + U1 y + U2 y^2 (reference: plane Couette (0.5, 0.5, 0),
 * source/coefficient.cu:149-159) and the precision of the transform path. */
typedef struct dns_params {
  int mx, my, mz;          /* padded x, padded span, 4*(Ny-1) */
  double n_pi_x, n_pi_y;   /* Lx = n_pi_x*pi, Lz = n_pi_y*pi */
  double Re, Ro, dt;
  double U0, U1, U2;
  int precision;           /* DNS_PREC_FP64 or DNS_PREC_MIXED */
  int device;              /* CUDA device ordinal */
} dns_params;

/* Step / IO records 4-6 of parameter.txt (include/parameters.h:16-27). */
typedef struct dns_run_params {
  int start_type, start_step, end_step, save_internal, save_recovery_internal;
  char output_file_prefix[512];
  char recovery_file_prefix[512];
} dns_run_params;

const char* dns_status_string(dns_status s);
const char* dns_last_error(void);
int dns_abi_version(void);

/* Reference defaults (problem::problem(), include/data.h:295-304 and
 * input/parameter.txt) with the Couette base flow. */
dns_status dns_params_default(dns_params* p);

/* Replaces RPCF_Paras::read_para (source/operation.cpp:115-138); unlike the
 * reference, a missing or short file is an error. */
dns_status dns_read_parameter_file(const char* path, dns_params* p, dns_run_params* rp);

/* Replaces problem(conf) + getDeviceInfo + allocDeviceMem + initFFT +
 * allocHostMemory (source/data.cpp:3-31, source/RPCFKernels.cu:17-128,
 * source/transform.cu:18-93, source/solver.cpp:216-257).  The operator
 * inverses (source/solver.cpp:260-320) are built on the device on the first
 * dns_bootstrap / dns_step. */
dns_status dns_create(const dns_params* p, dns_ctx** out);

/* No counterpart in the reference.  A batch of nruns independent runs of one
 * grid (runs[i] share mx, my, mz, box, base flow, precision and device; Re,
 * Ro and dt may differ): one context whose every pass is one launch for all
 * runs.  State and history arrays (dns_set_state, dns_get_state,
 * dns_set_history, dns_get_history) hold the runs one after another, H
 * pencils each; dns_step, dns_bootstrap, dns_step_profiled, dns_autotune
 * and dns_check_state act on all of them.  The entry points that take one
 * run's data (recovery files, initFlow, the per-function drop-ins of the
 * step, dns_solve_wall) refuse a batch.  nruns <= DNS_MAX_BATCH. */
#define DNS_MAX_BATCH 1024
dns_status dns_create_batch(const dns_params* runs, int nruns, dns_ctx** ctx);
dns_status dns_destroy(dns_ctx* ctx);

/* sizes: Nx, Ny, Nz, Kx, Px, Py, Pz, H (= Kx*Nz pencils) */
dns_status dns_geometry(const dns_ctx* ctx, int out[8]);
dns_status dns_get_stream(dns_ctx* ctx, void** cuda_stream);
dns_status dns_synchronize(dns_ctx* ctx);
/* bytes of device memory held by the context */
dns_status dns_memory_bytes(const dns_ctx* ctx, size_t* bytes);

/* ---- fused time step (the drop-in for nextStep) ---------------------- */

/* State in the reference's host layout: rhs_v / rhs_omega_y after a solve
 * (source/solver.cpp:95-96): [Nz][Kx] pencils of `pitch` bytes, Ny complex
 * doubles used per pencil, pencil (0,0) = u0 / w0.  where = DNS_HOST or
 * DNS_DEVICE.  Synchronous.  Setting the state keeps the AB2 history (as a
 * host-driven step of the reference does); call dns_bootstrap to restart it. */
dns_status dns_set_state(dns_ctx* ctx, const void* v, const void* omega, size_t pitch, int where);
dns_status dns_get_state(dns_ctx* ctx, void* v, void* omega, size_t pitch, int where);
/* The AB2 history: nonlinear terms at the Ny collocation points
 * (reference nonlinear_v / nonlinear_omega_y after a step). Synchronous. */
dns_status dns_get_history(dns_ctx* ctx, void* nv, void* nomega, size_t pitch, int where);
dns_status dns_set_history(dns_ctx* ctx, const void* nv, const void* nomega, size_t pitch, int where);

/* Failure detection (no counterpart in the reference): DNS_ERR_NONFINITE if
 * the current state or the AB2 history holds a NaN or an Inf, else DNS_OK.
 * One pass over state and history on the device (about 0.04 ms at
 * 256x129x256); synchronous. */
dns_status dns_check_state(dns_ctx* ctx);

/* Recovery file in the reference's format (source/output.cpp:105-178):
 * int mx, my, mz; size_t pSize, tSize (the reference's allocator sizes,
 * source/operation.cpp:152-180, pitches from cudaMalloc3D on this device);
 * Ny complex each of lambx0, lambz0, lambx0_p, lambz0_p, tv0, tomega_y_0;
 * tSize bytes each of rhs_v, rhs_v_p, rhs_omega_y, nonlinear_v,
 * nonlinear_omega_y in the pitched [Nz][Kx] pencil layout.  The "_p" fields
 * are written with the current values (a restart never reads them: the next
 * step replaces them before use).  Reading restores state and AB2 history
 * (the writer's pencil pitch is taken from tSize), after which dns_step
 * continues the run. */
dns_status dns_write_recovery(dns_ctx* ctx, const char* path);
dns_status dns_read_recovery(dns_ctx* ctx, const char* path);

/* output_velocity / write_velocity (source/output.cpp:19-103): the physical
 * velocity (u, v span, w wall-normal) and vorticity (omega_x, omega_y span,
 * omega_z wall-normal) of the current state on the padded grid, each
 * component as Py planes x my rows x mx doubles, unpitched, three components
 * per file.  Either path may be NULL.  Allocates its work buffers. */
dns_status dns_write_fields(dns_ctx* ctx, const char* velocity_path, const char* vorticity_path);

/* initFlow (source/RPCFKernels.cu:358-431): set the state to the reference's
 * analytic three-mode perturbation (amplitude 0.005), evaluated on mx x my
 * points and the Ny Gauss-Lobatto planes and taken to spectral space by the
 * forward transform without padding.  Like dns_set_state it leaves the AB2
 * history alone: call dns_bootstrap (the reference's "extra previous step")
 * before the first dns_step of a fresh run.  Allocates its work buffers. */
dns_status dns_init_flow(dns_ctx* ctx);

/* The "extra previous step" of source/main_loop.cpp:39-52: store the
 * nonlinear term of the current state as the AB2 history, so the first step
 * is forward Euler in the nonlinear term as in the reference. */
dns_status dns_bootstrap(dns_ctx* ctx);

/* nsteps x nextStep (source/solver.cpp:35-101): getUVW, transforms, Lamb
 * vector, rhsNonlinear, CN/AB2 right-hand sides, v solve, omega right-hand
 * side with the tilting term, omega solve -- one CUDA graph per step, no
 * host round trip. */
dns_status dns_step(dns_ctx* ctx, int nsteps);
/* No counterpart in the reference.  nsteps steps of each of n independent
 * runs (an ensemble: any grids, parameters and precisions), issued step by
 * step across the runs, each on its own context stream, so that the step
 * graphs of different runs execute concurrently and small grids share the
 * GPU.  Asynchronous like dns_step: synchronise each context (or the device)
 * before reading results.  A context may appear once. */
dns_status dns_step_many(dns_ctx* const* ctxs, int n, int nsteps);

/* No counterpart in the reference.  The bound, in SM clock cycles, after
 * which a staging wait of the mixed form's wall-normal passes gives up: the
 * CTA lets its copies in flight land, skips its work and the next
 * synchronising call reports DNS_ERR_TIMEOUT once (the flag is then cleared;
 * the state of that step is not valid).  Default 2^31 (about a second); a
 * negative value makes those waits give up at once, for tests of the timeout
 * path.  The next dns_step captures the step graph again. */
dns_status dns_set_wait_limit(dns_ctx* ctx, long long cycles);

/* Kernel variants and the autotuner (no counterpart in the reference).  A
 * tunable pass has several compiled kernels for the same arithmetic; the
 * context starts with the first variant, in the order listed below, that it
 * can run (the tensor-core y3 only by choice or by the autotuner).
 *   DNS_PASS_Y3: the backward wall-normal pass (getUVW + padded s2p)
 *     DNS_Y3_FFT     warp-synchronous FFTs of the even extensions, two lines
 *                    per warp (lengths with a warp plan);
 *     DNS_Y3_TENSOR  batched 3xTF32 Chebyshev products on the tensor cores
 *                    (tcgen05, FP32 accumulation): mixed form, Ny = 129;
 *     DNS_Y3_BLOCK   block-wide FFT (every grid).
 *   DNS_PASS_Y1: the forward wall-normal pass (p2s, nonlinear terms,
 *     right-hand sides): DNS_Y1_WARP (one warp per Lamb line, lengths with a
 *     warp plan) or DNS_Y1_BLOCK (every grid).
 *   DNS_PASS_ZB, DNS_PASS_ZF: the spanwise inverse / forward passes:
 *     DNS_Z_TENSOR_COPY  warp FFTs on tiles staged by tensor copies (mixed
 *                        form, Nz <= 256);
 *     DNS_Z_WARP         warp FFTs on tiles gathered through L1;
 *     DNS_Z_BLOCK        block-wide FFT (every grid).
 *   DNS_PASS_X: the streamwise pass (C2R, Lamb vector, R2C) on four rows
 *     per CTA: DNS_X_WARP3 (three warps, four lines each), DNS_X_WARP6 (six
 *     warps, two lines each) for lengths with warp plans, DNS_X_BLOCK (block
 *     FFT, every grid).
 *   DNS_PASS_Y2: the banded wall-normal solves; the block shape of the
 *     factor stream (ring stages x bytes per stage; the tilting table in
 *     shared memory or read through L1; the stream read with the L2
 *     evict-first policy or not): DNS_Y2_RING3_12K (table in shared memory),
 *     DNS_Y2_RING3_12K_EF (the same, evict-first), DNS_Y2_RING2_8K_EF,
 *     DNS_Y2_RING3_8K_EF.
 * dns_set_variant fails with DNS_ERR_ARG for a variant this context cannot
 * run.  dns_autotune times every available variant of every tunable pass
 * inside whole steps on this context's buffers and grid (state and AB2
 * history are saved and put back: the state is not modified), keeps the
 * fastest of each pass and, if ms is not NULL, writes the mean times in ms
 * to ms[pass * DNS_MAX_VARIANTS + variant] (-1 where unavailable).  It needs
 * a state (dns_set_state or dns_init_flow).  Synchronous; the next dns_step
 * captures the step graph again. */
enum {
  DNS_PASS_Y3 = 0,
  DNS_PASS_Y1 = 1,
  DNS_PASS_ZB = 2,
  DNS_PASS_ZF = 3,
  DNS_PASS_Y2 = 4,
  DNS_PASS_X = 5,
  DNS_NUM_PASSES = 6,
  DNS_MAX_VARIANTS = 4
};
enum { DNS_Y3_FFT = 0, DNS_Y3_TENSOR = 1, DNS_Y3_BLOCK = 2 };
enum { DNS_Y1_WARP = 0, DNS_Y1_BLOCK = 1 };
enum { DNS_Z_TENSOR_COPY = 0, DNS_Z_WARP = 1, DNS_Z_BLOCK = 2 };
enum { DNS_Y2_RING3_12K = 0, DNS_Y2_RING3_12K_EF = 1, DNS_Y2_RING2_8K_EF = 2, DNS_Y2_RING3_8K_EF = 3 };
enum { DNS_X_WARP3 = 0, DNS_X_WARP6 = 1, DNS_X_BLOCK = 2 };
dns_status dns_set_variant(dns_ctx* ctx, int pass, int variant);
dns_status dns_get_variant(const dns_ctx* ctx, int pass, int* variant);
dns_status dns_autotune(dns_ctx* ctx, double* ms);

/* The same steps without the graph, with CUDA events recorded around each
 * of the DNS_NUM_KERNELS kernels of a step on the context stream;
 * kernel_ms[k] = mean duration of kernel k (dns_kernel_name(k)).
 * Synchronous.  Replaces the reference's CURPCF_CUDA_PROFILING timers
 * (include/cuRPCF.h:14-15, source/nonlinear.cu:28-106). */
#define DNS_NUM_KERNELS 6
dns_status dns_step_profiled(dns_ctx* ctx, int nsteps, double kernel_ms[DNS_NUM_KERNELS]);
const char* dns_kernel_name(int k);

/* ---- reference-layout entry points (device pointers) ----------------- */

/* transform_3d_one (source/transform.cu:95-319): dir = DNS_BACKWARD maps
 * the spectral pencils (nz coefficients) to the physical field (the pencils
 * are overwritten, as in the reference); DNS_FORWARD maps the physical
 * field to pz coefficients per pencil.  pad = DNS_PADDING uses the pz
 * wall-normal points, DNS_NO_PADDING the nz points. */
dns_status dns_transform_3d_one(dns_ctx* ctx, int dir, void* phys, size_t pitch, void* spec,
                                size_t tpitch, int pad);
/* No counterpart in the reference.  dns_transform_3d_one for callers that
 * must not allocate device memory at call time (dns_transform_3d_one
 * cudaMallocs a work buffer on first use; an application that has reserved
 * nearly all device memory for itself, or a loop that cannot take the
 * implicit device synchronisation of cudaMalloc, cannot allow that).  Same
 * arguments and identical results; the work buffer is a 16 MiB static device
 * array per GPU, so one wall-normal plane of streamwise rows
 * (my * roundup(mx/2+1, 8) complex doubles) must fit, else DNS_ERR_ARG.
 * Calls on one device share that buffer: calls that overlap on the GPU race.
 * The first call on a device looks up the buffer's address; make it before
 * any stream capture. */
dns_status dns_transform_3d_one_noalloc(dns_ctx* ctx, int dir, void* phys, size_t pitch, void* spec,
                                        size_t tpitch, int pad);
/* transform (source/transform.cu:321-351): BACKWARD on six fields
 * (u, v, w, omega_x, omega_y, omega_z), FORWARD on three (lamb_z, lamb_y,
 * lamb_x order of the reference is immaterial). */
dns_status dns_transform(dns_ctx* ctx, int dir, int nfields, void* const* phys, size_t pitch,
                         void* const* spec, size_t tpitch);
/* cuda_transpose (source/transpose.cu:115-166); xyz is complex. */
dns_status dns_cuda_transpose(dns_ctx* ctx, int dir, void* xyz, size_t pitch, void* zxy,
                              size_t tpitch);
/* cheby_s2p / cheby_p2s (source/transform.cu:538-748), in place. */
dns_status dns_cheby_s2p(dns_ctx* ctx, void* zxy, size_t tpitch, int pad);
dns_status dns_cheby_p2s(dns_ctx* ctx, void* zxy, size_t tpitch, int pad);
/* getUVW (source/velocity.cu:22-170): reads f[2] (w) and f[5] (omega_z),
 * writes all six. */
dns_status dns_get_uvw(dns_ctx* ctx, void* const f[6], size_t tpitch);
/* computeLambVector (source/nonlinear.cu:307-428): out may alias in[0..2]. */
dns_status dns_compute_lamb(dns_ctx* ctx, void* const in[6], void* const out[3], size_t pitch);
/* rhsNonlinear (source/nonlinear.cu:130-242). */
dns_status dns_rhs_nonlinear(dns_ctx* ctx, void* lamb_x, void* lamb_y, const void* lamb_z,
                             size_t tpitch);
/* solveEq (source/solver.cpp:107-123): rhs <- inv * rhs for every pencil;
 * inv row-major [ky][kx][N][N] complex, rhs pitched pencils.  where =
 * DNS_DEVICE: both on the device, asynchronous.  where = DNS_HOST: both in
 * host memory, as the reference keeps them (source/solver.cpp:216-257);
 * streamed through a device staging buffer (allocated on first use),
 * synchronous. */
dns_status dns_solve_eq(dns_ctx* ctx, const void* inv, void* rhs, int N, size_t tpitch, int where);
/* solveEq (source/solver.cpp:107-123) for both wall-normal systems of every
 * pencil, without the explicit inverses: the banded factors of the time step
 * (built on first use) solve the reference's collocation systems
 * (source/coefficient.cu:7-86) exactly.  v and omega hold the right-hand
 * sides in the reference's layout ([Nz][Kx] pencils of tpitch bytes, Ny
 * complex used: v rows 0..3 wall values v(1), v(-1), v'(1), v'(-1), rows
 * 4..N values at y_2..y_{N-2}; omega rows 0..1 wall values, rows 2..N values
 * at y_1..y_{N-1}; pencil (0,0) the u0 / w0 systems) and are overwritten by
 * the Chebyshev coefficients of the solutions, as solveEq overwrites rhs.
 * No tilting term is added (that is part of the step's right-hand side).
 * Either pointer may be NULL: that system is not touched (the reference
 * solves v before it forms the omega_y right-hand side).  where = DNS_HOST
 * or DNS_DEVICE.  Synchronous; allocates its vectors (2 H Ny + 6 H complex)
 * on first use.  On device pencils with both systems the whole sequence
 * (right-hand-side preparation, DCT-I, integration, the banded solve of all
 * pencils in one launch, the wall polynomial added back) is one CUDA graph,
 * captured on the first call with those buffers and launched on each. */
dns_status dns_solve_wall(dns_ctx* ctx, void* v, void* omega, size_t tpitch, int where);
/* No counterpart in the reference.  Residual of solved systems: b the
 * collocation right-hand sides as dns_solve_wall takes them, x the
 * solutions it returned, A the reference's operators
 * (source/coefficient.cu:7-86).  out[0], out[1]: largest per-pencil
 * ||A x - b||_2 / ||b||_2 of the v and the omega systems; out[2], out[3]:
 * the same over all pencils together; out[4], out[5]: largest normwise
 * backward error ||A x - b||_inf / (||A||_inf ||x||_inf + ||b||_inf).
 * Synchronous; O(H Ny^2) on the device. */
dns_status dns_solve_residual(dns_ctx* ctx, const void* b_v, const void* b_omega, const void* x_v,
                              const void* x_omega, size_t tpitch, int where, double out[6]);
/* initAuxMatrix (source/solver.cpp:260-320): explicit inverses of the v and
 * omega operators of every pencil, row-major [ky][kx][nz][nz] complex. */
dns_status dns_init_aux_matrix(dns_ctx* ctx, void* inv_v, void* inv_omega, int where);
/* initAuxMatrix(pb, inversed = false): the operators themselves
 * (source/coefficient.cu:7-86), same layout; pencil (0,0) holds the
 * mean-mode operator in both.  Synchronous. */
dns_status dns_operator_matrices(dns_ctx* ctx, void* a_v, void* a_omega, int where);
/* The host tables initAuxMatrix fills (source/coefficient.cu:88-159):
 * T0, T2, T4 as [nz][nz] row-major (T_j and its 2nd / 4th derivative at the
 * Gauss-Lobatto point y_i = cos(pi i/(nz-1)) in entry [i][j]) and U, U', U''
 * at those points.  Host pointers; any may be NULL.  Synchronous. */
dns_status dns_operator_tables(dns_ctx* ctx, double* T0, double* T2, double* T4, double* U,
                               double* dU, double* ddU);

/* ---- the step function by function (reference-layout drop-ins) ----------
 * For callers that run the reference's own sequence (source/solver.cpp:
 * 35-101): get_rhs_v, solveEq(v), get_rhs_omega, solveEq(omega).  Pencils in
 * the reference's layout ([Nz][Kx] pencils of tpitch bytes, Ny complex used);
 * where = DNS_HOST (synchronous; staged through device vectors allocated on
 * first use) or DNS_DEVICE (asynchronous, in place).  dns_step does all of
 * it in one graph and is the fast path. */

/* getNonlinear + the worker's post-processing (source/nonlinear.cu:25-108,
 * source/rhs.cpp:83-127): from the state (v, omega_y coefficients) to the
 * nonlinear terms at the Ny collocation points, the reference's
 * nonlinear_v / nonlinear_omega_y; pencil (0,0) holds the raw lambda_x /
 * lambda_span values (lambx0 / lambz0).  Computed in the context's
 * precision; the context's own state and history are not touched.
 * Synchronous; allocates 4 H Ny complex on first use. */
dns_status dns_nonlinear(dns_ctx* ctx, const void* v, const void* omega, void* nv, void* nomega,
                         size_t tpitch, int where);
/* get_linear_v + the AB2 loop of get_rhs_v (source/linear.cpp:7-41,86-125,
 * source/rhs.cpp:185-219), every pencil but (0,0): rhs_v_p <- rhs_v (v^n);
 * rhs_v <- explicit CN v operator at y_2..y_{N-2} + dt (1.5 nv - 0.5 nv_p),
 * rows 0..3 zero.  FP64. */
dns_status dns_rhs_v(dns_ctx* ctx, void* rhs_v, void* rhs_v_p, const void* nv, const void* nv_p,
                     size_t tpitch, int where);
/* get_rhs_omega = get_linear_omega_y (source/linear.cpp:52-84,127-171),
 * every pencil but (0,0): rhs_omega <- explicit CN omega operator at
 * y_1..y_{N-1}, tilting -i beta U' dt/2 (rhs_v + rhs_v_p) with rhs_v = v^{n+1}
 * (after the v solve) and rhs_v_p = v^n, + dt (1.5 nomega - 0.5 nomega_p);
 * rows 0..1 zero.  FP64. */
dns_status dns_rhs_omega(dns_ctx* ctx, void* rhs_omega, const void* nomega, const void* nomega_p,
                         const void* rhs_v, const void* rhs_v_p, size_t tpitch, int where);
/* get_linear_zero_wave_u_w (source/linear.cpp:43-50,173-205): the mean-mode
 * right-hand sides, in place on u0 (tv0) and w0 (tomega_y_0), Ny complex
 * each, from lambda_x / lambda_span at the collocation points (lambx0,
 * lambz0) and their previous values. */
dns_status dns_rhs_mean(dns_ctx* ctx, void* u0, const void* lambx0, const void* lambx0_p, void* w0,
                        const void* lambz0, const void* lambz0_p, int where);

/* ---- slab decomposition plan (host only, no device work) --------------
 * No counterpart in the reference.  For R ranks: rank r owns the operator
 * slots kz' in [slot0, slot1) with both pencils kz' and Nz - kz' of each
 * (the per-pencil passes and the solve) and the wall-normal planes
 * [y0, y1) of the Py physical planes (the spanwise and streamwise passes).
 * out = {slot0, slot1, y0, y1, pencils owned}. */
dns_status dns_slab_ranges(int mx, int my, int mz, int nranks, int rank, int out[5]);
enum { DNS_SLAB_PENCILS = 0, DNS_SLAB_PLANES = 1 };
/* One block of an exchange: pencils p = kz * Kx + kx for kz in
 * [kz0, kz0 + nkz) and all kx (rows local_row0 .. of the pencil owner's
 * local buffer, which holds its runs in increasing kz), times the planes
 * [y0, y0 + ny) of the plane owner.  peer = the other rank. */
typedef struct {
  int peer, kz0, nkz, local_row0, y0, ny;
} dns_slab_segment;
/* The segments of this rank in role DNS_SLAB_PENCILS (its pencils, one
 * list per plane owner) or DNS_SLAB_PLANES (its planes, one list per pencil
 * owner), ordered by peer, then by kz: the backward exchange after the
 * first wall-normal pass sends each field's segments pencil owner -> plane
 * owner in that order, the forward exchange after the spanwise forward pass
 * sends them back.  seg may be NULL to get the count. */
dns_status dns_slab_segments(int mx, int my, int mz, int nranks, int rank, int role,
                             dns_slab_segment* seg, int cap, int* count);

/* ---- slab-decomposed step (one context per rank) ------------------------
 * No counterpart in the reference.  dns_slab_create makes rank `rank`'s
 * context of an R-rank decomposition (dns_slab_ranges): its pencil arrays
 * hold only its pencils, in local row order (the runs of
 * dns_slab_segments in increasing kz, Kx pencils per kz, Ny complex FP64
 * coefficients each), and the step runs in three parts with two exchanges
 * between them, which the caller performs (an all-to-all over NCCL, or
 * copies between the ranks' buffers on one device):
 *   DNS_SLAB_Y3: wall-normal backward pass on the rank's pencils; packs the
 *                six fields for every plane owner into `send`;
 *   exchange 0:  send -> the peers' recv, dns_slab_exchange_bytes(.., 0, ..)
 *                bytes per peer, buffers ordered by peer;
 *   DNS_SLAB_XZ: unpacks `recv`; spanwise inverse, streamwise (Lamb vector
 *                and rotation term) and spanwise forward passes on the
 *                rank's planes; packs the three fields for every pencil
 *                owner into `send`;
 *   exchange 1:  as exchange 0 with dns_slab_exchange_bytes(.., 1, ..);
 *   DNS_SLAB_Y1: unpacks `recv`; wall-normal forward pass and right-hand
 *                sides on the rank's pencils; with boot = 0 the banded
 *                solves of its slots (the new state).  boot = 1 runs the
 *                three parts as the bootstrap (the AB2 history only).
 * Per peer and field the packed buffers hold the segments in plan order,
 * each block [pencil][plane], in the transform precision (8 bytes per
 * complex value in the mixed form, 16 in FP64).  The parts are enqueued on
 * the context's stream (dns_get_stream) and return at once; `send` and
 * `recv` are device buffers the caller keeps until the work is done.
 * dns_synchronize reports device-side failures.  The whole-grid entry points
 * (dns_set_state, dns_step, ...) refuse a slab context. */
enum { DNS_SLAB_Y3 = 0, DNS_SLAB_XZ = 1, DNS_SLAB_Y1 = 2 };
enum { DNS_SLAB_V = 0, DNS_SLAB_OMEGA = 1, DNS_SLAB_NV = 2, DNS_SLAB_NOMEGA = 3 };
dns_status dns_slab_create(const dns_params* p, int nranks, int rank, dns_ctx** ctx);
/* send[peer], recv[peer]: bytes of exchange 0 or 1 (nranks entries each) */
dns_status dns_slab_exchange_bytes(const dns_ctx* ctx, int exchange, size_t* send, size_t* recv);
/* the rank's v, omega_y (DNS_SLAB_V, DNS_SLAB_OMEGA) or AB2 history
 * (DNS_SLAB_NV, DNS_SLAB_NOMEGA: Chebyshev coefficients of the nonlinear
 * terms) in local row order, np x Ny complex FP64, unpitched: into the
 * context (to_ctx = 1) or out of it.  Synchronous. */
dns_status dns_slab_local(dns_ctx* ctx, int which, void* buf, int where, int to_ctx);
dns_status dns_slab_part(dns_ctx* ctx, int part, int boot, void* send, const void* recv);

#ifdef __cplusplus
}
#endif
#endif /* DNS_B200_H */
