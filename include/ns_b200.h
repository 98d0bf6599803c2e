/*
 * ns_b200.h -- C ABI of the B200-native explicit right-hand side and SSP-RK3
 * time step of a 3D compressible Navier-Stokes finite-difference solver
 * (drop-in for the hot path of hamsteri15/3DNSsolver).
 *
 * Conventions
 *   - Every call returns ns_status; no C++ exception crosses this boundary and
 *     nothing calls exit().  ns_last_error_string() describes the last failure
 *     on the calling thread.
 *   - Host arrays at the boundary use the reference container layout
 *     (src/containers/array_4d.hpp:64-71): AoS [i][j][k][q], q fastest,
 *     dims (nx+6)(ny+6)(nz+6) x 5 doubles, 3 ghost cells per side
 *     (src/params.hpp:16-18).  Primitive order is [rho, p, u, v, w]
 *     (src/domain.hpp:49), conservative order [rho, rhoE, rhou, rhov, rhow]
 *     (src/domain.hpp:52).  Host pointers are borrowed for the call only.
 *   - One context per host thread; a context is not thread-safe.  All device
 *     work of a context is ordered on one CUDA stream (its own, or one adopted
 *     with ns_set_stream).
 *   - Device state is owned by the context (SoA FP64 with on-device halos).
 */
#ifndef NS_B200_H
#define NS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define NS_API __attribute__((visibility("default")))
#else
#define NS_API
#endif

#define NS_ABI_VERSION 1
#define NS_NGC 3 /* ghost cells per side, src/params.hpp:16-18 */
#define NS_NQ 5  /* variables per cell, src/domain.cpp:160 */

typedef enum ns_status {
    NS_OK = 0,
    NS_ERR_INVALID_ARG = 1,
    NS_ERR_OOM = 2,
    NS_ERR_CUDA = 3,
    NS_ERR_NONFINITE = 4,
    NS_ERR_TIMEOUT = 5,
    NS_ERR_UNSUPPORTED = 6,
    NS_ERR_NO_DEVICE = 7
} ns_status;

/* ConvectionScheme factory choices, src/driver.cpp:74-94 */
enum { NS_CONV_NONE = 0, NS_CONV_WENO5 = 1, NS_CONV_WENO5_CHAR = 2 };
/* WENO weight type, src/convection_schemes/weno-5.cpp:294,313 */
enum { NS_WEIGHTS_SHU = 0, NS_WEIGHTS_BORGES = 1 };
/* DiffusionScheme factory choices, src/driver.cpp:96-105 */
enum { NS_DIFF_NONE = 0, NS_DIFF_CENTERED = 1 };
/* Per-axis boundary: periodic (MPI_Cart periodic flag, src/decomposition.cpp:116-161)
 * or zeroth-order Neumann copy (src/boundary_conditions/boundary_neumann.cpp:22-132).
 * NS_BC_EXTERNAL (x axis only): the context is one slab of a domain split along x
 * (src/decomposition.cpp:116-143, one rank per GPU); its x ghost planes are the
 * neighbouring slabs' cells, which an exchange callback brings in before every
 * RK stage (src/communicator.cpp:16-57), see ns_set_exchange. */
enum { NS_BC_PERIODIC = 0, NS_BC_NEUMANN = 1, NS_BC_EXTERNAL = 2 };
/* Arithmetic of the stencil / flux / WENO work.  FP32 keeps the RK3
 * accumulation and all global reductions in FP64. */
enum { NS_PREC_FP64 = 0, NS_PREC_FP32 = 1 };
/* NS_SEM_REFERENCE reproduces the reference formulas exactly (including its
 * non-textbook terms); NS_SEM_PHYSICAL corrects them (no reference counterpart). */
enum { NS_SEM_REFERENCE = 0, NS_SEM_PHYSICAL = 1 };
/* Right-hand-side terms for ns_rhs */
enum { NS_TERM_CONVECTION = 1, NS_TERM_DIFFUSION = 2, NS_TERM_ALL = 3 };

/* Mirrors the hot-path fields of Params (src/params.hpp:20-43). */
typedef struct ns_params {
    int dim;             /* Geometry/Dim; dim != 3 skips the z convection sweep (weno-5.cpp:28) */
    int nx, ny, nz;      /* interior cells per axis */
    double Lx, Ly, Lz;   /* domain lengths; dx = Lx/nx (src/grid.cpp:12-19) */
    double mu, Pr, gamma;/* FluidProperties: constant viscosity, Prandtl, ratio of specific heats */
    double cfl;          /* Time/CFLmax */
    int convection;      /* NS_CONV_* */
    int weights;         /* NS_WEIGHTS_* */
    int diffusion;       /* NS_DIFF_* */
    int diffusion_order; /* 2, 4 or 6 (src/difference_operators/cd_constants.hpp) */
    int bc[3];           /* x (West/East), y (North/South), z (Back/Front): NS_BC_* */
    int precision;       /* NS_PREC_* */
    int semantics;       /* NS_SEM_* */
    int sensor;          /* 1: learned sensor gates the characteristic projection (FP32 only) */
    double sensor_threshold; /* sensor fires when sigmoid(logit) > threshold (default 0.5) */
    int check_finite;    /* 1: ns_advance, ns_time_step and ns_synchronize check the state and
                          * return NS_ERR_NONFINITE if an interior cell holds NaN/Inf or a
                          * non-positive density or pressure (the reference lets NaN propagate
                          * silently, src/time_scheme.cpp:104-117); 0 (default): no check */
    /* slab decomposition along x (bc[0] = NS_BC_EXTERNAL): */
    int slab_x0;         /* global index of this slab's first x cell */
    int slab_nx;         /* global cells along x (the slabs' nx sum to it) */
    int slab_periodic;   /* 1: the global x axis is periodic; 0: Neumann at the global ends
                          * (the end slabs fill their outer ghost planes themselves) */
    int sensor_period;   /* sensor = 1: evaluate the network every sensor_period steps and gate
                          * the steps in between with the same flags (0 or 1: every step) */
    int reserved[3];
} ns_params;

/* Global diagnostics of the device state (no reference counterpart: the
 * reference prints dt only, src/driver.cpp:61-64). */
typedef struct ns_diagnostics {
    long long steps;     /* steps taken by ns_advance / ns_time_step on this context */
    double dt;           /* dt of the last step (set_dt, src/time_scheme.cpp:127-136) */
    double next_dt;      /* dt the next step will use (CFL min over the current state) */
    double time;         /* sum of dt over the steps taken */
    double mass;         /* sum rho dV */
    double momentum[3];  /* sum rho u_d dV */
    double energy;       /* sum rhoE dV */
    double kinetic;      /* sum 0.5 rho |u|^2 dV */
    double enstrophy;    /* sum 0.5 rho |curl u|^2 dV (second-order central curl) */
    int nonfinite;       /* 1 if any interior conserved value is NaN/Inf */
    double sensor_fraction; /* fraction of faces the sensor flagged in the last stage */
} ns_diagnostics;

typedef struct ns_ctx ns_ctx;

NS_API const char* ns_status_string(ns_status s);
/* Message of the last failure on this thread ("" if none). */
NS_API const char* ns_last_error_string(void);
NS_API int ns_abi_version(void);

/* Fills *p with the defaults of the tutorial case (src/io/reader.cpp:3-172 fields). */
NS_API ns_status ns_params_default(ns_params* p);

/* Creates a context and allocates its device state on the current CUDA device.
 * Replaces Driver::run's construction of Grid/Domain/operators
 * (src/driver.cpp:9-25) for the hot path. */
NS_API ns_status ns_create(const ns_params* p, ns_ctx** out);
NS_API void ns_destroy(ns_ctx* ctx);
/* Adopts a caller's cudaStream_t.  NULL selects the context's own non-blocking
 * stream again (the legacy default stream cannot be adopted). */
NS_API ns_status ns_set_stream(ns_ctx* ctx, void* cuda_stream);
/* Number of elements of one host halo'd array: (nx+6)(ny+6)(nz+6)*5. */
NS_API size_t ns_host_array_elems(const ns_params* p);

/* ---- state transfer (host AoS with halos) -------------------------------- */
/* Sets the primitive state W (Domain::get_NS_primitive_array, src/domain.hpp:36). */
NS_API ns_status ns_upload_primitive(ns_ctx* ctx, const double* W);
NS_API ns_status ns_download_primitive(ns_ctx* ctx, double* W);
NS_API ns_status ns_download_conservative(ns_ctx* ctx, double* U);

/* ---- operator plug-ins (drop-in for the reference virtual interfaces) ----- */
/* ConvectionScheme::solve(grid, W, U, R) (src/convection_schemes/convection_scheme.hpp:26,
 * Weno5::solve src/convection_schemes/weno-5.cpp:3-37): R += convective residual.
 * W and U are read including their halos as given; only R's interior is written. */
NS_API ns_status ns_convection_solve(ns_ctx* ctx, const double* W, const double* U, double* R);
/* DiffusionScheme::solve(grid, comm, W, R) (src/diffusion_schemes/diffusion_scheme.hpp:14-17,
 * CenteredDiffusion::solve src/diffusion_schemes/centered_diffusion.cpp:3-68): R += viscous residual.
 * W is read including its halos as given. */
NS_API ns_status ns_diffusion_solve(ns_ctx* ctx, const double* W, double* R);
/* First RK stage's right-hand side from a primitive field: prim->cons on all cells,
 * boundary fill + halo exchange, cons->prim, R = 0, then the selected terms
 * (src/time_scheme.cpp:124-140).  W is read (halos included), R's interior written. */
NS_API ns_status ns_rhs(ns_ctx* ctx, const double* W, double* R, int terms);
/* TimeScheme::set_dt (src/time_scheme.cpp:98-136): CFL * min over interior cells. */
NS_API ns_status ns_compute_dt(ns_ctx* ctx, const double* W, double* dt_out);
/* TimeScheme::step (src/time_scheme.hpp:25-29, src/time_scheme.cpp:3-70): one SSP-RK3
 * step of host W (in/out) and U (out, may be NULL); dt_out receives the step's dt.
 * Host <-> device copies are part of the call.  When W (and U) lie in page-locked
 * host memory (cudaHostAlloc, or ns_host_register), an FP64 step on a single
 * domain overlaps the copies with the stages: W goes up in chunks of x-planes under
 * the first stage and comes down in chunks during the third.  The result is the
 * same bit for bit. */
NS_API ns_status ns_time_step(ns_ctx* ctx, double* W, double* U, double* dt_out);
/* Page-locks (cudaHostRegister) / releases a host range, for hosts that do not
 * link the CUDA runtime themselves, so that ns_time_step on arrays inside it
 * overlaps its copies.  No context needed; release before freeing the memory. */
NS_API ns_status ns_host_register(void* ptr, size_t bytes);
NS_API ns_status ns_host_unregister(void* ptr);

/* ---- device-resident time loop -------------------------------------------- */
/* Runs nsteps steps of TimeScheme::step on the device-resident state (the Driver
 * loop, src/driver.cpp:43-68, without host copies).  Asynchronous on the
 * context's stream; no host synchronisation inside, unless params.check_finite
 * is set: then the call waits for the steps and checks the state
 * (NS_ERR_NONFINITE, see ns_synchronize). */
NS_API ns_status ns_advance(ns_ctx* ctx, int nsteps);
/* dt of the last step and the sum of dt over the steps taken (0 before the
 * first step): TimeScheme::get_dt (src/time_scheme.hpp:31) plus the Driver's
 * time accumulation (src/driver.cpp:54-58).  Waits for the context's stream. */
NS_API ns_status ns_get_dt(ns_ctx* ctx, double* dt, double* time);
/* Blocks until the context's stream is idle.  NS_ERR_TIMEOUT if a bounded
 * device wait ran out since the context was created (a tensor-core wait of the
 * sensor's flag kernel, or a TMA tile wait of the FP64 face or viscous
 * kernels; the kernel then ended without its results).  With
 * params.check_finite set it then checks the current state: NS_ERR_NONFINITE if
 * an interior cell holds NaN/Inf or a non-positive density or pressure (the
 * message gives the number of such cells).  ns_time_step runs the same check
 * after its step. */
NS_API ns_status ns_synchronize(ns_ctx* ctx);
NS_API ns_status ns_get_diagnostics(ns_ctx* ctx, ns_diagnostics* out);
/* Kernel classes timed by ns_profile_step (NS_PROF_SENSOR: the per-step
 * sensor flags of the fused FP32 form; NS_PROF_XFACE_UPDATE: the FP64 x-faces
 * marched together with the cell update; NS_PROF_VISCOUS: the FP64 step's
 * viscous terms) */
enum { NS_PROF_STEP_BEGIN = 0, NS_PROF_FILL = 1, NS_PROF_FACE_X = 2, NS_PROF_FACE_Y = 3,
       NS_PROF_FACE_Z = 4, NS_PROF_UPDATE = 5, NS_PROF_STAGE_FUSED = 6, NS_PROF_SENSOR = 7,
       NS_PROF_XFACE_UPDATE = 8, NS_PROF_VISCOUS = 9, NS_PROF_N = 10 };
/* Runs one time step of the device-resident state with CUDA events recorded
 * between its kernels on the context's stream; ms[c] receives the device time
 * of kernel class c summed over the step, for c < n (n >= 7; classes at or
 * above n are left out of ms). */
NS_API ns_status ns_profile_step(ns_ctx* ctx, float* ms, int n);
/* ---- slab decomposition along x (multi-GPU) --------------------------------
 * Replaces the MPI halo exchange and dt reduction of the reference
 * (Communicator::communicate_x_direction, src/communicator.cpp:16-57, and the
 * MPI_Allreduce(MIN) of TimeScheme::set_dt, src/time_scheme.cpp:127-136) for a
 * context created with bc[0] = NS_BC_EXTERNAL.  The time-step calls
 * (ns_advance, ns_time_step) call the exchange callback on the context's stream
 * at two points of every step:
 *   what = NS_EXCHANGE_DT: before the first stage; the CFL minimum of this slab
 *     is in the 8 bytes at ns_slab_dt_slot (the bits of a positive double, or
 *     all ones if the slab has no finite value); the callback replaces it with
 *     the minimum over all slabs (as unsigned 64-bit integers);
 *   what = NS_EXCHANGE_HALO: before each of the three stages; the callback packs
 *     this slab's outer interior planes (ns_slab_pack), sends them to the
 *     neighbouring slabs, receives theirs and unpacks them into the ghost planes
 *     (ns_slab_unpack).  Sides at a non-periodic global end are filled by the
 *     library (Neumann) and need no exchange.
 * The callback enqueues all device work on the given stream (NCCL send/recv
 * on that stream, or host-staged copies) and returns NS_OK or an error, which
 * the step returns.  No kernel of the library waits on another slab. */
enum { NS_EXCHANGE_DT = 0, NS_EXCHANGE_HALO = 1 };
typedef ns_status (*ns_exchange_fn)(void* user, ns_ctx* ctx, int what, void* cuda_stream);
NS_API ns_status ns_set_exchange(ns_ctx* ctx, ns_exchange_fn fn, void* user);
/* Doubles of one packed side: 5 x 3 x ny x nz, order [q][layer][j][k]. */
NS_API size_t ns_slab_elems(ns_ctx* ctx);
/* Inside the NS_EXCHANGE_HALO callback: side 0 packs interior planes 0..2
 * (for the lower neighbour's upper ghost planes), side 1 planes nx-3..nx-1;
 * unpack writes ghost planes -3..-1 (side 0) or nx..nx+2 (side 1) of the
 * stage's input state.  dev_buf: ns_slab_elems doubles of device memory. */
NS_API ns_status ns_slab_pack(ns_ctx* ctx, int side, void* dev_buf);
NS_API ns_status ns_slab_unpack(ns_ctx* ctx, int side, const void* dev_buf);
/* Device address of the 8-byte CFL minimum slot (inside the NS_EXCHANGE_DT callback). */
NS_API ns_status ns_slab_dt_slot(ns_ctx* ctx, void** dev_ptr);

/* ---- learned troubled-face sensor (no reference counterpart) ----------------
 * An MLP 21 -> 32 -> 32 -> 1 (GELU) predicts from a face's stencil whether the
 * characteristic-wise WENO-5 flux differs from the component-wise one by more
 * than a relative threshold; with ns_params.sensor = 1 (FP32 characteristic
 * form, either semantics) the characteristic-wise flux is used only on the
 * faces the network flags and the component-wise flux elsewhere.  Time steps
 * evaluate the network on the state at the step's start (every sensor_period
 * steps); each stage then runs the component-wise stage on every face and
 * corrects the flagged faces by their characteristic-wise minus component-wise
 * flux (a compacted list).  The per-operator entry points (ns_convection_solve,
 * ns_rhs) evaluate it on the W they are given.  Parameters are
 * NS_SENSOR_NPARAMS floats: W1[32][32] (out, in; in >= 21 unused), b1[32],
 * W2[32][32], b2[32], w3[32], b3.  Device pointers below are caller-owned. */
#define NS_SENSOR_FEATURES 21
#define NS_SENSOR_NPARAMS 2145
/* Glorot-uniform weights and zero biases from a seed (host array). */
NS_API ns_status ns_sensor_init(unsigned long long seed, float* w);
/* Features (NS_SENSOR_FEATURES floats per face) and labels (0/1) of every face
 * of the context's current state along each convected axis, from FP64
 * component- and characteristic-wise fluxes; label = |f_char - f_comp|_2 >
 * rel_threshold (|f_char|_2 + 1e-12).  Appends nothing: rows 0..count-1 of the
 * device arrays are written; capacity is their row count.  The context's
 * state goes through one equation-of-state round trip (rounding level). */
NS_API ns_status ns_sensor_harvest(ns_ctx* ctx, float* d_features, float* d_labels,
                                   long long capacity, long long* count, double rel_threshold);
/* Adam (lr, beta 0.9/0.999) on the binary cross-entropy with logits, positive
 * class weighted by pos_weight, `epochs` passes over n samples in mini-batches
 * of `batch` (a seeded permutation per epoch).  w (host) is updated in place;
 * epoch_loss (host, may be NULL) receives the mean loss of each epoch.  BF16
 * tensor-core forward and backward with FP32 accumulation. */
NS_API ns_status ns_sensor_train(const float* d_features, const float* d_labels, long long n,
                                 int epochs, int batch, float lr, float pos_weight,
                                 unsigned long long seed, float* w, float* epoch_loss,
                                 void* cuda_stream);
/* Gradient (host, NS_SENSOR_NPARAMS) and mean loss of one batch of n samples. */
NS_API ns_status ns_sensor_gradients(const float* d_features, const float* d_labels, int n,
                                     float pos_weight, const float* w, float* grad, float* loss,
                                     void* cuda_stream);
/* Logits of n samples into d_logits. */
NS_API ns_status ns_sensor_predict(const float* d_features, long long n, const float* w,
                                   float* d_logits, void* cuda_stream);
/* Installs the network a sensor-gated context uses (host array; until called
 * the network is all zeros and never fires). */
NS_API ns_status ns_set_sensor_weights(ns_ctx* ctx, const float* w);

/* ---- convection residual without device allocation -------------------------
 * No counterpart in the reference.  For callers that may not allocate device
 * memory or have it allocated for them: hosts that serve all device memory
 * from their own pool and give a plugin no allocation budget, and real-time
 * loops that cannot take cudaMalloc's latency, its device synchronisation or
 * an out-of-memory failure mid-run.  Same result as ns_convection_solve
 * (R += convective residual, halos of W and U read as given) but W, U and R
 * are DEVICE pointers, each to 5 consecutive planes (q = 0..4) of the halo'd
 * box (nx+6) x (ny+6) x (nz+6) doubles with k fastest; work is queued on
 * cuda_stream (NULL: the legacy default stream) and the call returns without
 * waiting.  The face fluxes live in one array of NS_NOALLOC_SCRATCH_BYTES
 * compiled into the library; grids whose face fluxes do not fit (beyond about
 * 64^3 cells in FP64) are rejected with NS_ERR_INVALID_ARG.  The array is
 * reserved on a device when the library's device code is loaded there, which
 * under CUDA's default lazy loading can be the first call of this entry point
 * on that device, and stays reserved until the process exits: make one call
 * at start-up (or set CUDA_MODULE_LOADING=EAGER) so that no later call can
 * fail for want of memory, and make that first call before any stream capture
 * begins.  Every call looks up the array's address in the current context.
 * All calls on a device share the array: calls that overlap on the GPU race,
 * so serialise them.  Nothing is allocated: no cudaMalloc, no cudaFree, no
 * allocating library call. */
#define NS_NOALLOC_SCRATCH_BYTES (32u << 20)
NS_API ns_status ns_convection_solve_noalloc(const ns_params* p, const double* W, const double* U,
                                             double* R, void* cuda_stream);
/* Measured FMA throughput of the current device in TFLOP/s (2 flops per FMA):
 * fp64 = 1 for double, 0 for float.  The denominator of the compute roofline
 * of the FMA-bound WENO kernels (no counterpart in the reference). */
NS_API ns_status ns_fma_peak(int fp64, double* tflops);
/* Self-test of the bounded device waits every TMA and tensor-core kernel uses:
 * one block waits, at most `polls` polls, on an mbarrier phase that nothing
 * completes.  *ran_out = 1 when the wait gave up and reported (the correct
 * outcome), 0 if it claimed completion; *ms = the wait's device time.  The
 * device stays usable afterwards (no fault, no trap).  No reference
 * counterpart. */
NS_API ns_status ns_wait_selftest(unsigned polls, int* ran_out, double* ms);
/* Self-test of the FP64 arithmetic written out in the kernels on `n` seeded
 * random pairs: max_ulp[0] = the largest distance, in units in the last place,
 * of the WENO quotient (Newton-Raphson reciprocal from the hardware estimate
 * with a Markstein correction) from the IEEE quotient; max_ulp[1] = that of
 * the sound-speed 1/sqrt (Newton-Raphson) from CUDA's rsqrt.  max_ulp points
 * to two values.  No reference counterpart. */
NS_API ns_status ns_div_selftest(long long n, unsigned long long seed, unsigned long long* max_ulp);
/* Device kernels launched by this context since creation (for launch accounting). */
NS_API long long ns_kernel_launches(ns_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* NS_B200_H */
