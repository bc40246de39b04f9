/*
 * spectral_b200 C-ABI -- the drop-in boundary of the B200 pseudo-spectral
 * Navier-Stokes path.
 *
 * Every entry point takes plain pointers and sizes, returns an int status
 * (0 = success, negative = error; sns_last_error() describes the last
 * failure of the calling thread) and never throws or exits.  Field arrays are
 * device pointers to interleaved complex numbers in the reference layout
 * n = i + nx*j + nx*ny*k, x fastest (src/Scalar.cpp:683), either complex64
 * (prec = SNS_C64) or complex128 (prec = SNS_C128).  `stream` is a
 * cudaStream_t passed as void* (NULL = the legacy default stream); work is
 * queued on it asynchronously unless a function says it synchronises.
 * Dimensions must be powers of two up to 4096 per axis for the transforms.
 *
 * The reference (smsolivier/spectral_upcxx) is a C++ library; its callers use
 * the Scalar / Vector / Operators / FFT1D classes.  Those classes are provided
 * with unchanged signatures by spectral_upcxx_b200/api/*.H on top of this
 * ABI, so the ABI is what an FFI (ctypes, cgo, JNI) binds.  Each declaration
 * names the reference code it replaces.
 */
#ifndef SPECTRAL_B200_H
#define SPECTRAL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SNS_C64 0  /* complex64: FP32 bulk arithmetic */
#define SNS_C128 1 /* complex128: FP64, the reference's precision (src/FFT1D.H:13) */

#define SNS_OK 0
#define SNS_ERR_ARG (-1)
#define SNS_ERR_UNSUPPORTED (-2)
#define SNS_ERR_CUDA (-3)
#define SNS_ERR_ALLOC (-4)
#define SNS_ERR_TIMEOUT (-5)

/* flags of sns_fft3d */
#define SNS_FFT_NORMALISE 1   /* multiply by 1/(nx ny nz) (Scalar::inverse, src/Scalar.cpp:223-227) */
#define SNS_FFT_ZERO_NYQUIST 2 /* zero the i=nx/2, j=ny/2, k=nz/2 planes (Scalar::zeroHighModes, src/Scalar.cpp:336-370) */

/* ---- status ---------------------------------------------------------- */
/* Text of the calling thread's last error ("" if none).  Replaces the
 * print-and-exit ERROR macro (src/Scalar.cpp:9-13) below the C++ API. */
const char* sns_last_error(void);
int sns_version(void);

/* ---- device memory (caching pool) ------------------------------------ */
/* Stream-ordered caching allocator for field storage.  Replaces
 * upcxx::new_array / delete_array in Scalar::init and ~Scalar
 * (src/Scalar.cpp:38-40, 95, 117).  sns_free returns the block to the pool;
 * a later sns_malloc may hand it out again for work on the same stream. */
int sns_malloc(void** ptr, size_t bytes);
int sns_free(void* ptr);
int sns_pool_trim(void);
int sns_memcpy_h2d(void* dst, const void* src, size_t bytes, void* stream);
int sns_memcpy_d2h(void* dst, const void* src, size_t bytes, void* stream);
/* deep copy (Scalar copy constructor / operator=, src/Scalar.cpp:52-66) */
int sns_memcpy_d2d(void* dst, const void* src, size_t bytes, void* stream);
int sns_memset(void* ptr, int value, size_t bytes, void* stream);
int sns_stream_synchronize(void* stream);
/* precision conversion of n complex values (either direction or a copy) */
int sns_convert(void* dst, int dst_prec, const void* src, int src_prec, int64_t n,
                void* stream);

/* ---- transforms -------------------------------------------------------- */
/* In-place unnormalised 3D DFT of one field.  dir = -1 forward
 * (exp(-2 pi i jk/n)), +1 inverse -- the sign convention of
 * Scalar::transform (src/Scalar.cpp:400-646; FFT1D::transform's DIR,
 * src/FFT1D.cpp:95-101).  flags: SNS_FFT_NORMALISE | SNS_FFT_ZERO_NYQUIST. */
int sns_fft3d(void* field, int64_t nx, int64_t ny, int64_t nz, int dir, int flags, int prec,
              void* stream);
/* The same transform over up to 12 fields of equal shape in one batch. */
int sns_fft3d_many(void* const* fields, int nfields, int64_t nx, int64_t ny, int64_t nz,
                   int dir, int flags, int prec, void* stream);
/* Choose the plan of sns_fft3d / sns_fft3d_many for nfields fields of
 * nx*ny*nz by measurement (the counterpart of the reference's FFTW_MEASURE
 * planning, src/FFT1D.cpp:18-22): per axis the tile width, thread count and
 * radix order (radix-16 stages with the remainder last or first, or radix-8
 * stages), for each axis the TMA-staged form of the pass (one or two
 * shared-memory stages per persistent CTA), and for 128 x 128 planes the
 * plane pass against two line passes.
 * Runs on scratch fields from the pool; the choice is cached per device and
 * shape and used by every later transform of that shape (results agree with
 * the default plan to rounding).  SNS_TUNE=1 tunes each new shape on first use. */
int sns_fft3d_tune(int64_t nx, int64_t ny, int64_t nz, int nfields, int prec, void* stream);
/* Check of the transforms queued so far on this device (no reference
 * counterpart: the reference's FFTW calls have no asynchronous failure).
 * The TMA-staged passes of a tuned plan bound every wait; one that runs out,
 * or a tile box that fails the kernel's own alignment check, is recorded on
 * the device.  Synchronises `stream`, reads and clears the record:
 * SNS_ERR_TIMEOUT (results of those transforms invalid) or SNS_OK. */
int sns_fft3d_check(void* stream);
/* The line passes of selected axes only (bit 0: x, bit 1: y, bit 2: z), in that
 * order, the last one multiplied by `scale` (1: none).  The local phases of the
 * slab-distributed transform of Scalar::transform (src/Scalar.cpp:419-566: the
 * y and x lines of the rank's own z planes, then the z lines of the planes
 * gathered by the transpose). */
int sns_fft3d_axes(void* field, int64_t nx, int64_t ny, int64_t nz, int axes, int dir,
                   double scale, int prec, void* stream);
/* Scalar::forward(): transform(-1) + zeroHighModes (src/Scalar.cpp:208-215). */
int sns_forward(void* field, int64_t nx, int64_t ny, int64_t nz, int prec, void* stream);
/* Scalar::inverse(): transform(+1) then divide by N (src/Scalar.cpp:217-229). */
int sns_inverse(void* field, int64_t nx, int64_t ny, int64_t nz, int prec, void* stream);
/* Batched in-place 1D DFTs: `howmany` lines of n elements `stride` apart,
 * line b starting at element b*dist.  Backs FFT1D::transform(ptr, N, stride,
 * DIR) and FFT1D::init/transform(ptr, DIR) (src/FFT1D.cpp:14-101), which
 * run one strided line per FFTW call; unnormalised. */
int sns_fft1d_many(void* data, int64_t n, int64_t stride, int64_t howmany, int64_t dist,
                   int dir, int prec, void* stream);
/* The same lines, each multiplied by `scale` after its transform: FFT1D::inverse
 * (src/FFT1D.cpp:60-67) is dir = +1 with scale = 1/n (exact for the power-of-two
 * n supported here, so equal to the reference's division by n). */
int sns_fft1d_many_scaled(void* data, int64_t n, int64_t stride, int64_t howmany, int64_t dist,
                          int dir, double scale, int prec, void* stream);

/* ---- spectral operators (Fourier-space fields) ------------------------ */
/* Scalar::zeroHighModes (src/Scalar.cpp:336-370). */
int sns_zero_high_modes(void* field, int64_t nx, int64_t ny, int64_t nz, int prec,
                        void* stream);
/* Scalar::gradient: g_d = i k_d f (src/Scalar.cpp:245-276). */
int sns_gradient(const void* f, void* gx, void* gy, void* gz, int64_t nx, int64_t ny,
                 int64_t nz, int prec, void* stream);
/* Scalar::laplacian: -|k|^2 f (src/Scalar.cpp:278-306). */
int sns_laplacian(const void* f, void* out, int64_t nx, int64_t ny, int64_t nz, int prec,
                  void* stream);
/* Scalar::laplacian_inverse(a, b): f /= (a - b|k|^2) where |k|^2 != 0
 * (src/Scalar.cpp:308-334). */
int sns_laplacian_inverse(void* f, double a, double b, int64_t nx, int64_t ny, int64_t nz,
                          int prec, void* stream);
/* Vector::curl: i k x v (src/Vector.cpp:92-122). */
int sns_curl(const void* const v[3], void* const out[3], int64_t nx, int64_t ny, int64_t nz,
             int prec, void* stream);
/* Vector::divergence: sum_d i k_d v_d (src/Vector.cpp:124-153). */
int sns_divergence(const void* const v[3], void* out, int64_t nx, int64_t ny, int64_t nz,
                   int prec, void* stream);
/* Vector::laplacian: -|k|^2 v_d (src/Vector.cpp:155-181). */
int sns_vector_laplacian(const void* const v[3], void* const out[3], int64_t nx, int64_t ny,
                         int64_t nz, int prec, void* stream);
/* Vector::cross (src/Vector.cpp:66-90): inverse-transform copies of both
 * Fourier operands, complex point-wise a x b, forward transform with Nyquist
 * zeroing.  out may alias neither input.  Uses 6 fields of pooled scratch. */
int sns_cross(const void* const a[3], const void* const b[3], void* const out[3], int64_t nx,
              int64_t ny, int64_t nz, int prec, void* stream);
/* Vector::cross without any device allocation (no counterpart in the
 * reference).  For callers that cannot let the library call cudaMalloc --
 * device memory fully reserved by another allocator, or a loop that must not
 * enter the driver's allocation path -- the six work fields and the twiddle
 * tables live in a static array of the library (24 MiB of work space plus
 * 192 KiB of tables), which each GPU that uses this function holds until the
 * process exits.  Boxes of at most 262144 complex128 or 524288 complex64
 * points (64^3 / 64^2*128) are accepted; larger ones return SNS_ERR_ARG, and
 * other bad arguments return what sns_cross returns for them.  The first call
 * on a device sets up the array (its device address is looked up, which is
 * also when the driver creates it on that GPU): make that call before another
 * allocator reserves the device memory, where it could fail for lack of
 * memory, and before any stream capture.  All calls share the array and it
 * keeps the last call's contents: calls that overlap on the GPU (different
 * streams at once) race, so serialise them.  Results agree with sns_cross's
 * to rounding (its twiddle tables are generated on the device). */
int sns_cross_noalloc(const void* const a[3], const void* const b[3], void* const out[3],
                      int64_t nx, int64_t ny, int64_t nz, int prec, void* stream);
/* Scalar::average: mean of |f_i| over n values, accumulated in FP64
 * (src/Scalar.cpp:15-22).  Synchronises `stream`; the result is written to
 * the host double *out. */
int sns_average_abs(const void* f, int64_t n, int prec, double* out, void* stream);

/* ---- element-wise Operators (src/Operators.cpp:9-99) ------------------ */
/* out = alpha*x + beta*y; y may be NULL (out = alpha*x).  Covers Scalar and
 * Vector +, -, and double*Scalar / double*Vector. */
int sns_axpby(double alpha, const void* x, double beta, const void* y, void* out, int64_t n,
              int prec, void* stream);
/* out = a*b element-wise (Scalar operator*, src/Operators.cpp:9-19). */
int sns_mul(const void* a, const void* b, void* out, int64_t n, int prec, void* stream);

/* ---- fused Navier-Stokes stepper (exec/ns.cpp:132-217) ---------------- */
typedef struct sns_ns sns_ns;
/* Create a stepper for an nx*ny*nz box with viscosity nu and time step dt
 * (ns.cpp:43-46).  Allocates its state and work fields (12 fields). */
int sns_ns_create(sns_ns** handle, int64_t nx, int64_t ny, int64_t nz, double nu, double dt,
                  int prec, void* stream);
/* The same stepper for a real velocity field (no reference counterpart; the
 * reference transforms real data as complex, src/Scalar.cpp:400-646): it keeps
 * the half spectrum kx = 0 .. nx/2-1 (the kx = nx/2 plane is zero after
 * zeroHighModes, and kx < 0 is the complex conjugate), so every pass moves
 * half the bytes; the x transforms become real-to-complex / complex-to-real.
 * Its functions take and return full Fourier fields exactly as for
 * sns_ns_create; inputs must be Hermitian (Fourier transforms of real fields).
 * nx must be a power of two >= 32.  Closures are not available on it. */
int sns_ns_create_real(sns_ns** handle, int64_t nx, int64_t ny, int64_t nz, double nu, double dt,
                       int prec, void* stream);
int sns_ns_destroy(sns_ns* handle);
/* Start from Fourier V0 and omega0 = curl V0: the Pi0 projection and the
 * Forward-Euler first step (ns.cpp:132-153).  Device pointers in the
 * stepper's precision. */
int sns_ns_bootstrap(sns_ns* handle, const void* const V0[3], const void* const omega0[3]);
/* Set the AB2 state directly: Fourier V1 and cross0 (= V0 x omega0). */
int sns_ns_set_state(sns_ns* handle, const void* const V1[3], const void* const cross0[3]);
/* Advance nsteps AB2 / projection / Crank-Nicolson steps (ns.cpp:167-217),
 * queued on the stepper's stream without host synchronisation.  After the
 * first step the step's launches are captured once as a CUDA graph (on a
 * private stream) and replayed; environment SNS_GRAPH=0 at creation keeps
 * direct launches.  Changing the closure drops the captured graph. */
int sns_ns_step(sns_ns* handle, int nsteps);
/* Copy out V1, omega1 = curl V1 and cross0 (any pointer may be NULL). */
int sns_ns_get_state(sns_ns* handle, void* const V1[3], void* const omega1[3],
                     void* const cross0[3]);
/* Diagnostics of the velocity after the last step, accumulated in FP64:
 * the divergence monitor div.average() (ns.cpp:209-210), kinetic energy
 * 0.5<|u|^2>, enstrophy 0.5<|omega|^2> and max |div u_hat|.  Synchronises. */
int sns_ns_stats(sns_ns* handle, double* div_avg, double* energy, double* enstrophy,
                 double* max_div);
/* The same four values (div_avg, energy, enstrophy, max_div) queued on the
 * stepper's stream and copied to out4 (pinned host or device memory) without
 * waiting: a run can read its monitor every step (ns.cpp:206-210) while the
 * GPU keeps stepping, and look at the values once the stream has been
 * synchronised.  No reference counterpart (the reference's div.average()
 * returns synchronously, src/Scalar.cpp:15-22).  Unlike sns_ns_stats it does
 * not check the stepper's error word; sns_ns_check does. */
int sns_ns_stats_async(sns_ns* handle, double* out4);
/* Synchronise and report whether any step since the last check hit a bounded
 * wait of the persistent xy pass or of the TMA-staged z pass that gave up
 * (SNS_ERR_TIMEOUT: the results
 * of those steps are invalid).  sns_ns_stats performs this check too. */
int sns_ns_check(sns_ns* handle);
/* Number of kernel launches one sns_ns_step(h, 1) issues in steady state (a
 * plan whose update pass carries the next step's z-inverse pass launches one
 * more in the first step after a bootstrap or a new state). */
int sns_ns_launches_per_step(sns_ns* handle);
/* Tune the stepper's plan by measurement (no reference counterpart; the
 * reference's planning is FFTW_MEASURE per line plan, src/FFT1D.cpp:18-22):
 * times candidate tile shapes of each pass -- K1 z-inverse + curl tile (direct
 * loads, or TMA-staged with one or two stages), the
 * y passes' run width, thread count and radix order, the x pass's rows per
 * CTA (direct or TMA-staged), the update pass's width, then the L2 prefetch
 * distance of all passes
 * (SNS_PF=0..4 in the environment fixes it) -- on the stepper's own fields (seeded data
 * for the timing, zero again after) and keeps the fastest per pass.  Call it after create and before the first
 * bootstrap, set_state or step (SNS_ERR_ARG otherwise); the choice is cached
 * per device and box shape, so later steppers of the same shape reuse it
 * without measuring.  SNS_TUNE=1 in the environment makes every sns_ns_create
 * tune.  Tuned and untuned steppers agree to rounding. */
int sns_ns_tune(sns_ns* handle);
/* The stepper's plan as text (no reference counterpart; the reference's
 * planning is FFTW_MEASURE per line plan, src/FFT1D.cpp:18-22): the pass
 * structure and tile shapes chosen for this box, e.g.
 * "passes=5 xy=separate k1=8x1(tma1) y=W16/T256/16-first zW=16 xG=4(tma) pf=0 tuned".  Writes at most len bytes
 * (NUL-terminated) to buf; returns the full length. */
int sns_ns_describe(sns_ns* handle, char* buf, int len);
/* Per-pass timing (no reference counterpart; the reference times phases with
 * CH_Timer, src/Scalar.cpp:421-617).  While enabled, every step records CUDA
 * events between its passes on the stepper's stream; enabling clears the
 * totals.  sns_ns_pass_times synchronises and returns, per pass, the summed
 * milliseconds and the number of timed launches (arrays of `max` entries);
 * the return value is the number of passes per step, or a negative error. */
int sns_ns_profile(sns_ns* handle, int enable);
int sns_ns_pass_times(sns_ns* handle, double* total_ms, int* launches, int max);

/* ---- eddy-viscosity closure of the stepper ---------------------------------
 * No reference counterpart (exec/ns.cpp has no subgrid model).  With a
 * closure set, every step adds the divergence of tau_ij = 2 nu_t S_ij to the
 * nonlinear term cross1 (ns.cpp:203-206) before the unchanged AB2 /
 * projection / Crank-Nicolson update; S_ij and the model inputs come from the
 * velocity gradient A_ij = d_j u_i (real parts).  Models: SNS_CLOSURE_NONE
 * (the plain step), SNS_CLOSURE_SMAGORINSKY (nu_t = cs_delta2 sqrt(2 S:S),
 * cs_delta2 = (Cs Delta)^2), SNS_CLOSURE_MLP (nu_t from the packed MLP at
 * `mlp`, device memory that must outlive the steps).  kc > 0 restricts the
 * run to the modes |k| <= kc (the LES cutoff: the nonlinear term, velocity
 * and history of the modes beyond it are set to zero every step; with
 * SNS_CLOSURE_NONE it applies to the plain step).  Needs nx*ny*nz to be a
 * multiple of 32 for a model; allocates six more work fields on first use. */
#define SNS_CLOSURE_NONE 0
#define SNS_CLOSURE_SMAGORINSKY 1
#define SNS_CLOSURE_MLP 2
int sns_ns_set_closure(sns_ns* handle, int model, double cs_delta2, const void* mlp, double kc);
/* Spectral weight of the closure's eddy-stress divergence: mode k receives it
 * times clamp((|k| - k_lo) / (k_hi - k_lo), 0, 1), a ramp from k_lo to k_hi
 * (k_hi <= k_lo: a sharp split, every |k| > k_lo at full weight; the default
 * k_lo = k_hi = 0 applies it to every mode).  The damping then acts on the
 * small resolved scales, as in a variational multiscale split, while nu_t
 * (MLP or Smagorinsky) still comes from the full resolved gradient.  No
 * reference counterpart. */
int sns_ns_set_sgs_band(sns_ns* handle, double k_lo, double k_hi);

/* ---- learned closure: MLP 9 -> 64 -> 64 -> 1 on the tensor cores ----------
 * No reference counterpart.  FP32 master parameters (nparams floats: W1[64][16]
 * with columns 9..15 zero, b1[64], W2[64][64], b2[64], w3[64], b3) and a packed
 * inference copy (packed_bytes: bf16 W1, W2, w3; f32 b1, b2, b3, s_in, s_out).
 * Inputs are 16 bf16 per sample (s_in * A_ij in row-major order, zero padded);
 * nu_t = s_out * softplus(z), ReLU hidden layers, FP32 accumulation. */
int sns_mlp_sizes(int64_t* nparams, int64_t* packed_bytes);
int sns_mlp_pack(const float* master, double s_in, double s_out, void* packed, void* stream);
/* nut[M] = the model at the M rows of X (device pointers, 16-byte aligned),
 * on the tcgen05 tensor cores (128 points per tile, accumulators in tensor
 * memory). */
int sns_mlp_infer(const void* packed, const void* X, int64_t M, float* nut, void* stream);
/* Tracer particles: one move of np particles (Particle::move,
 * src/Particle.cpp:12-46, for the whole population of exec/ns.cpp:157-203 at
 * once).  loc: np x 3 doubles (x, y, z) in [0, 2 pi], updated in place; vel:
 * np x 3 doubles receiving the interpolated velocity (Particle::m_v; NULL to
 * skip); u: the three PHYSICAL velocity fields (after the inverse transform;
 * real parts are used), nx, ny, nz >= 2.  Cell index, trilinear weights, sum
 * order and wrap are the reference's; with complex128 fields the positions
 * equal the reference's bit for bit.  Device pointers. */
int sns_particles_move(double* loc, double* vel, int64_t np, const void* const u[3], int64_t nx,
                       int64_t ny, int64_t nz, int prec, double K, void* stream);
/* Synchronises the device; SNS_ERR_TIMEOUT (and clears the record) if a
 * tensor-core MLP kernel stopped waiting for its MMAs since the last call,
 * else SNS_OK.  No reference counterpart. */
int sns_mlp_status(void);
/* Gradient of the mean weighted squared error w (softplus(z) - target)^2
 * (target in model units, i.e. nu_t / s_out; weight NULL = 1) over B samples
 * (rows idx[0..B) of X, target and weight, or rows 0..B when idx is NULL).
 * grad: nparams + 1 floats (gradients, then the mean loss), device memory.
 * X and the packed model 16-byte aligned; runs on the tcgen05 tensor cores
 * (persistent CTAs, weight gradients accumulated in tensor memory).
 * Synchronises the stream. */
int sns_mlp_grad(const void* packed, const void* X, const float* target, const float* weight,
                 const int* idx, int64_t B, float* grad, void* stream);
/* One Adam step (bias correction for step >= 1) on the masters; refreshes
 * the packed copy's weights and biases. */
int sns_mlp_adam(float* master, float* m, float* v, const float* grad, int step, double lr,
                 double beta1, double beta2, double eps, void* packed, void* stream);

/* ---- filtered-DNS data for the closure -------------------------------------
 * Cubic grids, powers of two.  Fourier fields follow the reference's
 * unnormalised convention, so a coarse copy is scaled by nc^3 / nf^3. */
/* Sharp spherical cutoff |k| <= kc of nfields fine fields onto nc^3 grids. */
int sns_spectral_truncate(const void* const* in, void* const* out, int nfields, int64_t nf,
                          int64_t nc, double kc, int prec, void* stream);
/* Zero-padded copy of coarse fields on nf^3 grids (modes |k_d| < nc/2). */
int sns_spectral_pad(const void* const* in, void* const* out, int nfields, int64_t nc, int64_t nf,
                     int prec, void* stream);
/* Training pairs from one fine Fourier velocity V (nf^3): X (nc^3 rows of 16
 * bf16: s_in times the filtered gradient) and nut (nc^3 floats: the pointwise
 * least-squares eddy viscosity -(tau^d : S) / (2 S : S) of the filtered SGS
 * stress tau_ij = filter(u_i u_j) - filter(ubar_i ubar_j), products formed on
 * the fine grid); optionally the weight S : S of each pair (the stress
 * residual |tau^d + 2 nu S|^2 is 4 S:S (nu - nut)^2 plus a constant) and the
 * filtered coarse velocity Vc. */
int sns_sgs_sample(const void* const V[3], int64_t nf, int64_t nc, double kc, double s_in,
                   int prec, void* X, float* nut, float* weight, void* const Vc[3], void* stream);
/* E[k] = sum over the shell round(|k|) = k of |V_hat|^2 / (2 N^2), k < nshell
 * (device doubles), so that sum_k E[k] = <|u|^2> / 2. */
int sns_energy_spectrum(const void* const V[3], int64_t nx, int64_t ny, int64_t nz, int prec,
                        double* E, int nshell, void* stream);

/* ---- batched ensemble of NS boxes ----------------------------------------
 * No reference counterpart: the reference runs one box per process
 * (exec/ns.cpp).  An ensemble holds independent boxes of up to 8 distinct
 * sizes (powers of two in [16, 256] per axis), each with its own viscosity,
 * sharing dt and precision; every box follows the ns.cpp:132-217 sequence
 * exactly as sns_ns does.  One ensemble step is five launches, one per stage,
 * each over every box; SNS_ENS_GRAPH replays them as one captured CUDA graph,
 * SNS_ENS_EAGER launches them directly, SNS_ENS_SEQUENTIAL steps the boxes one
 * after another with the single-box stepper's kernels (a baseline). */
typedef struct sns_ens sns_ens;
#define SNS_ENS_GRAPH 0
#define SNS_ENS_EAGER 1
#define SNS_ENS_SEQUENTIAL 2
/* dims: 3 per box (nx, ny, nz); nu: one per box.  tune != 0 times the
 * candidate tile configurations of every stage on the ensemble (zeroed
 * fields) and keeps the fastest; tune = 0 takes the first that fits. */
int sns_ens_create(sns_ens** handle, int nboxes, const int64_t* dims, const double* nu, double dt,
                   int prec, int tune, void* stream);
int sns_ens_destroy(sns_ens* handle);
/* Number of boxes. */
int sns_ens_boxes(sns_ens* handle);
/* Per-box counterparts of sns_ns_bootstrap / set_state / get_state. */
int sns_ens_bootstrap(sns_ens* handle, int box, const void* const V0[3],
                      const void* const omega0[3]);
int sns_ens_set_state(sns_ens* handle, int box, const void* const V1[3],
                      const void* const cross0[3]);
int sns_ens_get_state(sns_ens* handle, int box, void* const V1[3], void* const omega1[3],
                      void* const cross0[3]);
/* Advance every box nsteps steps (mode: SNS_ENS_GRAPH, _EAGER, _SEQUENTIAL),
 * queued on the ensemble's stream. */
int sns_ens_step(sns_ens* handle, int nsteps, int mode);
/* Diagnostics of every box after the last step, 4 doubles per box in the
 * order of sns_ns_stats (div_avg, energy, enstrophy, max_div).  Synchronises. */
int sns_ens_stats(sns_ens* handle, double* out);
/* The configuration of each stage: threads per CTA, line-run cap, persistent
 * grid (3 ints per stage into out[max]).  Returns the number of stages. */
int sns_ens_tuning(sns_ens* handle, int* out, int max);
/* Run nsteps ensemble steps with CUDA events between the stages (the state
 * advances); ms[5] receives the mean milliseconds of each stage.  Synchronises
 * and returns the number of stages. */
int sns_ens_stage_times(sns_ens* handle, int nsteps, double* ms);
/* Kernel launches per ensemble step in the given mode. */
int sns_ens_launches_per_step(sns_ens* handle, int mode);

#ifdef __cplusplus
}
#endif

#endif
