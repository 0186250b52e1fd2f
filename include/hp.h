/*
 * hp.h -- C ABI of the B200 (sm_100a) Fokker-Planck propagation library for
 * densities on SO(3) x R^n (n = 2 or 3).
 *
 * Each entry point replaces one MEX gateway or MATLAB function of the reference
 * (fdcl-gwu/hybridPendulum-UP); the citation is on each declaration.  All
 * entry points return an int status (HP_OK == 0); hp_last_error() gives a
 * message for the last failure on the calling thread.
 *
 * Array arguments use the reference's MATLAB layouts (column-major, complex
 * values interleaved re/im as in the R2018a MEX API):
 *   F  (2lmax+1, 2lmax+1, lmax+1, 2Bx, 2Bx[, 2Bx])  complex, F(m+lmax+1, n+lmax+1, l+1, i, j, k)
 *   f  (2B, 2B, 2B, 2Bx, 2Bx[, 2Bx])                real (or complex), f(alpha, beta, gamma, i, j, k)
 *   MR (2lmax+1, 2lmax+1, lmax+1, n)                complex
 * with lmax = B-1.  `mem` says where a pointer lives (HP_DEVICE or HP_HOST);
 * host pointers are staged through the plan's device workspace.  A host F
 * input that is 16-byte aligned and page-locked and mapped into the device
 * address space over its whole extent (e.g. cudaHostAlloc / cudaMallocHost, or
 * a torch pin_memory tensor) is instead read in place by the layout kernel,
 * which reads only the entries the plan keeps (|m|, |n| <= l, and m >= 0 for
 * HP_REAL: about a fifth of the full array at B = 15); hp_host_read_in_place
 * tells which.  Either way the call returns after the input has been read.
 */
#ifndef HP_H
#define HP_H

#ifdef __cplusplus
extern "C" {
#endif

enum hp_status {
  HP_OK = 0,
  HP_ERR_INVALID = 1,     /* null pointer, bad enum, bad size            */
  HP_ERR_SHAPE = 2,       /* sizes inconsistent with the plan            */
  HP_ERR_ALLOC = 3,       /* device or host allocation failed            */
  HP_ERR_CUDA = 4,        /* a CUDA call failed                          */
  HP_ERR_UNSUPPORTED = 5, /* input outside the supported model class     */
  HP_ERR_NONFINITE = 6,   /* a NaN/Inf guard fired                       */
  HP_ERR_NO_MODEL = 7,    /* propagation requested before hp_plan_set_model */
  HP_ERR_MASS_DRIFT = 8   /* the l = 0 mass guard of hp_state_set_guard fired */
};

enum hp_precision {
  HP_FP64 = 0,  /* every kernel in FP64                                           */
  HP_MIXED = 1  /* FP32 operators / transforms, FP64 coefficient accumulation     */
};

enum hp_symmetry {
  HP_REAL = 0,    /* coefficients of a real density: only m >= 0 rows are stored,
                     m < 0 follow from F^l_{-m,-n}[-k] = (-1)^(m-n) conj F^l_{mn}[k] */
  HP_COMPLEX = 1  /* general complex coefficients: every (l, m, n) row is stored     */
};

enum hp_method { HP_EULER = 0, HP_MIDPOINT = 1, HP_RK2 = 2, HP_RK4 = 3 };
enum hp_mem { HP_DEVICE = 0, HP_HOST = 1 };

typedef struct hp_plan hp_plan;
typedef struct hp_state hp_state;

/* Sizes of a plan (all counts are elements, bytes are device bytes). */
typedef struct {
  int B, lmax, Bx, N, ndim, precision, symmetry;
  long long nx;          /* (2Bx)^ndim                                    */
  long long nrows;       /* stored (l, m, n) rows                         */
  long long n_full;      /* elements of the full MATLAB F layout          */
  long long n_grid;      /* elements of the f grid: (2B)^3 * nx           */
  long long state_bytes; /* device bytes of one resident coefficient state */
} hp_plan_info_t;

/*
 * Pendulum model: the derivative inputs of the reference MEX
 * pendulum_propagate(F,X,OJO,MR,bt,G,dt,L,u,CG,method)
 * (propagation/mex/sources/pendulum_propagate/kernel.cu:16-76).
 *   L      omega-grid period: x_i = -L/2 + L*j/(2Bx)            (pendulum.m:90-99)
 *   b      damping: Omega-dot contains -b_i Omega_i               (pendulum.m:424-427)
 *   G      noise matrix G = H H^T / 2, row-major 3x3 (ndim x ndim used)  (pendulum.m:202-208)
 *   gyro   J^-1(-Omega x J Omega) for diagonal J written as
 *          (gyro0*O2*O3, gyro1*O1*O3, gyro2*O1*O2)             (pendulum.m:145-158)
 * X and OJO of the MEX are functions of (L, J) and are rebuilt from them;
 * u and CG are plan tables.  MR is passed to hp_plan_set_model.
 */
typedef struct {
  double L;
  double b[3];
  double G[9];
  double gyro[3];
} hp_model;

/* Plan: tables (Wigner-d, quadrature weights, Clebsch-Gordan, twiddles) are
 * built on the device in FP64.  Replaces the per-call setup of every MEX
 * (e.g. propagation/mex/sources/fftSO3R/kernel.cu:20-130) and the MATLAB table
 * builders Wigner_d.m:1-47, getu.m:132-163, clebsch_gordan.m:1-43.
 * B: 2..32 (2B-point Euler grids); Bx: 2..32 (2Bx-point omega axes).  FFT
 * lengths whose prime factors are 2, 3 and 5 (2B, 2Bx in 4, 6, 8, 10, 12,
 * 16, 18, 20, 24, 30, 32, 36, 40, 48, 50, 54, 60, 64) run the fastest
 * kernels; other lengths use a direct DFT for their larger prime factor.
 * The derivative takes 3-D grids of up to 32 points per axis. */
int hp_plan_create(hp_plan** plan, int B, int Bx, int ndim, int precision, int symmetry);
int hp_plan_destroy(hp_plan* plan);
int hp_plan_get_info(const hp_plan* plan, hp_plan_info_t* info);
/* *in_place = 1 when a host F input of `bytes` bytes at `ptr` is read in place
 * (16-byte aligned, page-locked and mapped into the current device's address
 * space at its first and last byte), 0 when it is copied whole to the device
 * first. */
int hp_host_read_in_place(const void* ptr, long long bytes, int* in_place);
/* Stream for every launch of this plan (a cudaStream_t; NULL = legacy default). */
int hp_plan_set_stream(hp_plan* plan, void* cuda_stream);
const char* hp_last_error(void);

/* Measurement hooks (no counterpart in the reference, whose only timing is
 * tic/toc around each loop step, pendulum.m:270,314).  hp_plan_profile(1)
 * starts bracketing every kernel launch of the plan with CUDA events on the
 * plan's stream, grouped by kernel family; hp_plan_profile_get(i, ...) returns
 * family i's name, summed device time and launch count (HP_ERR_INVALID past
 * the last family).  hp_plan_launch_count counts every kernel launched by the
 * plan since creation. */
int hp_plan_profile(hp_plan* plan, int enable);
int hp_plan_profile_get(hp_plan* plan, int i, char* name, int name_cap, double* total_ms,
                        long long* count);
int hp_plan_launch_count(hp_plan* plan, long long* count);

/* Engine of the forward transform's beta contraction, the stage
 * F^l_mn[w] = sum_b w_b d^l_mn(beta_b) Q_b[m][n][w] of fftSO3R.m:89-106 (the
 * per-degree cuTENSOR contractions of the MEX, fftSO3R/kernel.cu:130-180).
 * HP_BETA_AUTO: the tensor cores (tcgen05, three TF32 products per FP32
 * product) in HP_MIXED plans with B >= 15, CUDA-core FMAs otherwise (FP64
 * plans always); HP_BETA_SIMT: CUDA-core FMAs; HP_BETA_TENSOR: the tensor cores
 * in every HP_MIXED plan; HP_BETA_TENSOR_BF16: the tensor cores with BF16x3
 * operands (each operand split into three BF16 parts, six BF16 products per
 * FP32 product, FP32 accumulation) in every HP_MIXED plan.  hp_plan_tc_errors returns the number of
 * tensor-core thread blocks of the plan whose bounded wait on the tensor core
 * gave up since the previous call (their outputs are not valid; the transform
 * itself still returns HP_OK, so poll this where it matters; 0 in normal
 * operation); the call synchronises the device and resets the count. */
enum hp_beta_engine { HP_BETA_AUTO = 0, HP_BETA_SIMT = 1, HP_BETA_TENSOR = 2, HP_BETA_TENSOR_BF16 = 3 };
int hp_plan_set_beta_engine(hp_plan* plan, int engine);
int hp_plan_tc_errors(hp_plan* plan, int* count);

/* Launch-shape tuning (no counterpart in the reference).  The knobs are the
 * runtime launch shapes of the transforms: synth_pt, the omega points per item
 * of the synthesis beta stage (1, 2 or 4; FP32 plans), synth_waves, the
 * resident waves of synthesis blocks (how many omega chunks a block walks),
 * tc_waves, the waves of tensor-core CTAs of the forward beta contraction, and
 * tc_form, its kernel (1: the warp-specialised pipeline fed by TMA tensor
 * copies, 0: the staged single-warpgroup kernel).
 * hp_plan_autotune times every candidate on scratch of the plan's sizes (one
 * coefficient state and one grid density, allocated and freed by the call)
 * with CUDA events on the plan's stream, keeps the fastest, and records it in
 * a process-wide cache keyed by (B, Bx, ndim, precision, symmetry, beta
 * engine); plans created (or given a beta engine) later with the same key
 * start from the cached shapes.  backward_ms / forward_ms (may be NULL)
 * receive the best median transform times (forward: 0 when the forward
 * transform does not use the tensor cores).  hp_tune_cache_save/load write
 * and read the cache as a text file, one key and its shapes per line.
 * hp_plan_set_tune sets knobs by hand (0 keeps a knob, -1 for tc_form). */
int hp_plan_autotune(hp_plan* plan, double* backward_ms, double* forward_ms);
int hp_plan_set_tune(hp_plan* plan, int synth_pt, int synth_waves, int tc_waves, int tc_form);
int hp_plan_get_tune(const hp_plan* plan, int* synth_pt, int* synth_waves, int* tc_waves, int* tc_form);
int hp_tune_cache_save(const char* path);
int hp_tune_cache_load(const char* path);

/* Model for the propagation entry points.  MR: complex (2lmax+1,2lmax+1,lmax+1,ndim)
 * in the full layout; only its degree-1, m2=0 block may be non-zero (the
 * gravity term of pendulum.m:166-192 depends on R through R^T e3 only);
 * otherwise HP_ERR_UNSUPPORTED. */
int hp_plan_set_model(hp_plan* plan, const hp_model* model, const double* MR, int mem);

/* Copy of the plan's Wigner-d table d(2lmax+1, 2lmax+1, lmax+1, 2B) in the
 * layout of pendulum.m:107-111 (d(m+lmax+1, n+lmax+1, l+1, j)); out is FP64. */
int hp_wigner_d(hp_plan* plan, double* d, int mem);
/* Quadrature weights w(2B) of fftSO3R.m:62-66. */
int hp_quad_weights(hp_plan* plan, double* w, int mem);

/* Forward transform F = fftSO3R(f): replaces fftSO3R_mex('forward', f, d, w)
 * (propagation/mex/sources/fftSO3R/kernel.cu:11-195) and fftSO3R.m:89-106.
 * f real (HP_REAL plans) or complex interleaved (HP_COMPLEX plans). */
int hp_fftSO3R_forward(hp_plan* plan, const double* f, double* F, int mem);
/* Backward transform f = ifftSO3R(F): replaces fftSO3R_mex('backward', F, d)
 * (kernel.cu:196-391), ifftSO3R.m:16-37 and the inline pendulum.m:284-304. */
int hp_fftSO3R_backward(hp_plan* plan, const double* F, double* f, int mem);

/* One propagation step Fnew = integrate(Fold): replaces
 * pendulum_propagate (ndim=3, propagation/mex/sources/pendulum_propagate/kernel.cu:9-519)
 * and pendulum_propagate_reduced (ndim=2, .../pendulum_propagate_reduced/kernel.cu:9-262),
 * i.e. the integrate/derivative pair of pendulum.m:346-527 and
 * pendulum_reduced.m:320-465.  method: HP_EULER/MIDPOINT/RK2/RK4. */
int hp_pendulum_propagate(hp_plan* plan, const double* Fold, double* Fnew, double dt,
                          int method, int mem);
/* The derivative dF of pendulum.m:388-527 / pendulum_reduced.m:362-465. */
int hp_pendulum_derivative(hp_plan* plan, const double* F, double* dF, int mem);

/* Density-side gravity model of the reduced pendulum: the inputs of the MEX
 * pendulum_propagate_reduced_den(F,f,X,mR,bt,G,dt,L,u,d,w,method)
 * (propagation/mex/sources/pendulum_propagate_reduced_den/kernel.cu:9-325,
 * integrate.cu:220-445) and of pendulum_reduced_den.m:401-533.  The gravity
 * term is formed on the grid, FMR_i = fftSO3R(f . mR_i), instead of by the
 * Clebsch-Gordan product.  model: L, b, G as for hp_plan_set_model (gyro
 * unused).  mR: real (2, 2B, 2B, 2B), component fastest (MATLAB layout of
 * pendulum_reduced_den.m:132).  Needs ndim = 2 and HP_REAL; replaces any model
 * set by hp_plan_set_model (and is replaced by it). */
int hp_plan_set_den_model(hp_plan* plan, const hp_model* model, const double* mR, int mem);
/* One step of the density-gravity model.  f: the real grid density of Fold,
 * (2B,2B,2B,2Bx,2Bx), used by the first derivative evaluation; NULL recomputes
 * it from Fold by the backward transform (the later stages always do so, as
 * integrate.cu of the reference MEX and pendulum_reduced_den.m:359-399). */
int hp_pendulum_propagate_den(hp_plan* plan, const double* Fold, const double* f, double* Fnew,
                              double dt, int method, int mem);

/* Gyro-bias attitude model: the inputs of the MEX
 * gyrobias_propagate(F,X,dt,u,G1,G2)
 * (propagation/mex/sources/gyrobias_propagate/kernel.cu:8-130) and of the
 * integrate function of gyro_bias.m:226-300.  The state is (R, x) with x the
 * 3-D gyro bias on the grid x_i = -L/2 + L*j/(2Bx) (gyro_bias.m:57-66 has
 * L = 2), and
 *   dF = -sum_i F_omega[x_i f]^l (u^l_i)^T            bias drift (226-265)
 *        + sum_ij G1_ij F^l (u^l_i)^T (u^l_j)^T        gyro random walk (268-279)
 *        + sum_ij G2_ij c_ij F                         bias random walk (281-297)
 * with c_ij the diffusion multipliers of hp_model for period L (the reference
 * writes them with pi = 2 pi / L at L = 2).  G1, G2: row-major 3x3, host.
 * Needs ndim = 3; replaces any other model of the plan (and is replaced by
 * hp_plan_set_model / hp_plan_set_den_model).  hp_pendulum_propagate,
 * hp_pendulum_derivative and the state API then run this model; the adjoint
 * entry points return HP_ERR_UNSUPPORTED for it. */
int hp_plan_set_gyro_bias_model(hp_plan* plan, double L, const double* G1, const double* G2);
/* Fnew = Fold + dt dF (the Euler step of gyro_bias.m:299 and the MEX). */
int hp_gyrobias_propagate(hp_plan* plan, const double* Fold, double* Fnew, double dt, int mem);

/* ---- reverse mode (no counterpart in the reference) ----
 * Gradients of a scalar loss L(F_T) of a forward-Euler trajectory
 * F_{n+1} = F_n + dt A F_n (hp_pendulum_propagate with HP_EULER), with the
 * convention dL = Re sum conj(lam) dF over the full layout (the convention of
 * torch complex gradients).  For HP_REAL plans gradients are those on the
 * real-density subspace: lamT is first projected onto it and lam0 lies in it. */
typedef struct {
  double b[3];       /* dL/db_i                                                */
  double G[9];       /* dL/dG_ij (row-major; G_ij and G_ji enter through one term) */
  double gyro[3];    /* dL/dgyro_i (ndim = 3)                                  */
  double gscale[3];  /* dL/ds_i at s = 1, where MR_i -> s_i MR_i (a J_i^-1 scale) */
} hp_model_grad;
/* out = A^H lam (the exact adjoint of hp_pendulum_derivative), full layout. */
int hp_pendulum_derivative_adjoint(hp_plan* plan, const double* lam, double* out, int mem);
/* Reverse pass of nsteps Euler steps from F0: lam0 = dL/dF0 and the model
 * gradients.  The trajectory is recomputed from checkpoints taken every
 * checkpoint_every steps (device memory: ceil(nsteps/k) + k states).
 * method must be HP_EULER; lam0 or grad may be NULL. */
int hp_pendulum_adjoint(hp_plan* plan, const double* F0, const double* lamT, int nsteps, double dt,
                        int method, int checkpoint_every, double* lam0, hp_model_grad* grad, int mem);

/* Derivative without allocation: the same dF as hp_pendulum_derivative, for
 * callers that must not allocate device memory while they run (a propagation
 * loop on a GPU whose memory another framework owns through its own allocator,
 * or an estimator working inside a fixed, pre-reserved memory budget), where a
 * cudaMalloc in the middle of a step can fail, fragment the pool or stall on a
 * device-wide synchronisation.  No counterpart in the reference.
 *   F, dF   device pointers, full MATLAB layout (as for hp_pendulum_derivative).
 * All scratch lives in one static device array of HP_NOALLOC_SCRATCH_BYTES
 * that every GPU loading the library keeps until the process exits; problems
 * needing more return HP_ERR_SHAPE.  Per stored coefficient row and omega point
 * it takes 64 bytes (FP64) or 48 bytes (mixed) on a 3-D omega grid, 48 / 40
 * bytes on a 2-D grid, plus the plane tile list: about 0.5 M (FP64) / 0.7 M
 * (mixed) such points in 3-D, 0.7 M / 0.8 M in 2-D.  It covers omega grids of
 * up to 32 points per axis (2Bx in 4..32; larger grids return
 * HP_ERR_UNSUPPORTED whatever their size) and the coefficient-gravity models
 * of hp_plan_set_model (a density-gravity model returns HP_ERR_UNSUPPORTED).
 * The plan and its model
 * must exist already (hp_plan_create / hp_plan_set_model allocate).  The first
 * call on a device looks up the array's device address, so make that first call
 * before any stream capture.  Every call shares the one array: calls that may
 * overlap on the GPU (other streams, other threads) race and must be ordered by
 * the caller.  Runs on the plan's stream and returns without synchronising. */
#define HP_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
int hp_pendulum_derivative_noalloc(hp_plan* plan, const double* F, double* dF);

/* Real-harmonic transforms of real functions on SO(3) alone (no omega axes),
 * batched over nbatch independent functions on the plan's SO(3) grid (the
 * plan's omega part is not used):
 *   hp_fftSO3_real_forward  replaces  F = fftSO3(f, B, true)  (fftSO3.m:61-119)
 *   hp_fftSO3_real_backward replaces  f = ifftSO3(F, true)    (ifftSO3.m:24-84)
 * f: real (2B, 2B, 2B, nbatch), f(alpha, beta, gamma, b); F: real
 * (2lmax+1, 2lmax+1, lmax+1, nbatch) in the real basis built from Wigner-d by
 * the Psi table of fftSO3.m:62-88.  FP64 for every plan precision.  Callers:
 * the SO(3)-only models (gyro_nobias.m) and fftSO3_deriv.m, whose derivative
 * dF = sum_i eta_i F (u_i)^T uses getu(lmax, true) (getu.m:45-107). */
int hp_fftSO3_real_forward(hp_plan* plan, const double* f, double* F, int nbatch, int mem);
int hp_fftSO3_real_backward(hp_plan* plan, const double* F, double* f, int nbatch, int mem);
/* Product rule in the real basis, fftSO3_prod(func1, func2, B, true)
 * (fftSO3_prod.m:97-205): FG from real F, G (2lmax+1, 2lmax+1, lmax+1, batch).
 * Computed as Re T FG_c T^H with FG_c the complex product (hp_fftSO3_prod) of
 * F_c = T^H F T, G_c = T^H G T, T^l the unitary of fftSO3_prod.m:103-120. */
int hp_fftSO3_real_prod(hp_plan* plan, const double* F, const double* G, double* FG, int batch, int mem);

/* Product rule of fftSO3_prod.m:209-265 (complex branch), batched over `batch`
 * independent pairs: FG^l = sum (2l1+1)(2l2+1)/(2l+1) [CG^T (F^l1 kron G^l2) CG]_l.
 * F, G, FG: (2lmax+1, 2lmax+1, lmax+1, batch) complex. */
int hp_fftSO3_prod(hp_plan* plan, const double* F, const double* G, double* FG, int batch,
                   int mem);

/* ---- hybrid collision operator (2-D reduced model and 3-D Omega, FP64 tables) ----
 * hp_collision_create builds the one-time tables of the reference's
 *   [lambda,indR,PC] = getLambda_mex(R,x,dWall,h,r,theta_t,lambda_max,false)
 *     (propagation/discrete/mex/sources/pendulum_reduced_collision/src/getLambda.cu:8-85)
 *   Omega_new = getOmega_mex(R,x,indR,epsilon,PC,'new')      (.../src/getOmega.cu:8-103)
 *   [fcL,fcL_indx] = getFcL_mex(x,Omega_new,lambda,Gd,nD)    (.../src/getFcL.cu:11-166)
 * on the plan's SO(3) grid and its omega grid of period L (callers:
 * propagation/pendulum_reduced_hybrid.m:130-142).  *numR receives the number
 * of colliding attitudes.  hp_collision_df is
 *   df = pendulum_reduced_discrete_propagate(true,f,lambda,indR,fcL,fcL_indx)
 *     (.../src/mexPropagate.cpp:6-77, propagate.cu:6-121; caller pendulum_reduced_hybrid.m:232)
 * with f, df real grid densities f(a,b,c,i,j).  hp_collision_tables copies the
 * tables out in the MEX layouts: lambda [ix][k], indR [k] (0-based), omega
 * [ix][k][ndim], fcL and fcL_indx [ix][k][d], PC [iR][3]; NULL skips a table.
 * On a 3-D plan (no reference counterpart: getOmega.cu:86-96 takes
 * Omega = [x1, x2, 0]) the operator uses all three components: omega = R Omega
 * in the switching rate and the reset map, Omega+ in R^3 and a 3-D Gaussian
 * landing kernel of covariance Gd (3x3); ix = i + 2Bx j + 4Bx^2 k, at most
 * 32768 omega points (16-bit tap indices).  hp_state_hybrid_step accepts
 * a coefficient-gravity model (hp_plan_set_model) as well as the density-
 * gravity model, so a 3-D plan runs the 3-D hybrid loop. */
typedef struct hp_collision hp_collision;
typedef struct {
  double d, h, r;          /* wall distance, pivot-to-tip height, tip radius */
  double theta_t;          /* half width of the switching ramp (rad)       */
  double lambda_max;       /* maximum switching rate                       */
  double epsilon;          /* coefficient of restitution                   */
  double L;                /* omega-grid period                            */
  double Gd[9];            /* reset-noise covariance, column-major ndim x ndim
                              in the first ndim^2 entries                  */
  int nD;                  /* taps kept per landing point (<= 32)          */
} hp_collision_params;
int hp_collision_create(hp_plan* plan, const hp_collision_params* params, hp_collision** coll, int* numR);
int hp_collision_destroy(hp_collision* coll);
int hp_collision_tables(hp_collision* coll, double* lambda, int* indR, double* omega, double* fcL,
                        short* fcL_indx, double* PC, int mem);
int hp_collision_df(hp_collision* coll, const double* f, double* df, int mem);
/* The table builders one MEX call at a time, for callers that build, keep or
 * reload the tables separately as pendulum_reduced_hybrid.m:130-141 does (it
 * caches fcL in a .mat file).  Tables use the layouts of hp_collision_tables;
 * all of lambda/indR/omega/fcL/fcL_indx/PC live in `mem`.
 *   hp_collision_lambda  replaces [lambda,indR,PC] = getLambda_mex(R,x,d,h,r,theta_t,lambda_max,false)
 *     (.../src/getLambda.cu:8-85, mexLambda.cpp:78-94): uses d, h, r, theta_t,
 *     lambda_max, L of params; *numR receives the number of colliding
 *     attitudes; lambda ([ix][k], nx * numR), indR and PC ([iR][3]) may each be
 *     NULL (call once with NULL to size them).
 *   hp_collision_omega   replaces Omega_new = getOmega_mex(R,x,indR,epsilon,PC,'new')
 *     (.../src/getOmega.cu:8-59, 73-92): Omega+ [ix][k][ndim] of the numR
 *     attitudes indR (ascending, 0-based; others are rejected); uses epsilon, L.
 *   hp_collision_fcL     replaces [fcL,fcL_indx] = getFcL_mex(x,Omega_new,lambda,Gd,nD)
 *     (.../src/getFcL.cu:11-166): the nD largest Gaussian taps per landing
 *     point, normalised per source point, times lambda dx^n; uses Gd, nD, L.
 *   hp_collision_create_from_tables builds the operator of hp_collision_df and
 *     hp_state_hybrid_step from given tables, the inputs of
 *     pendulum_reduced_discrete_propagate(true,f,lambda,indR,fcL,fcL_indx)
 *     (.../src/mexPropagate.cpp:6-77); the tables are copied, fcL_indx entries
 *     outside [0, nx) or indR not ascending in [0, (2B)^3) give HP_ERR_INVALID.
 *     hp_collision_tables then returns lambda, indR, fcL and fcL_indx only. */
int hp_collision_lambda(hp_plan* plan, const hp_collision_params* params, int* numR, double* lambda, int* indR,
                        double* PC, int mem);
int hp_collision_omega(hp_plan* plan, const hp_collision_params* params, int numR, const int* indR, double* omega,
                       int mem);
int hp_collision_fcL(hp_plan* plan, const hp_collision_params* params, int numR, const double* omega,
                     const double* lambda, double* fcL, short* fcL_indx, int mem);
int hp_collision_create_from_tables(hp_plan* plan, int numR, int nD, const int* indR, const double* lambda,
                                    const double* fcL, const short* fcL_indx, int mem, hp_collision** coll);

/* ---- initial densities ----
 * Matrix Fisher x Gaussian on the plan's grid, the initial condition of
 * propagation/pendulum.m:210-220 (and pendulum_reduced*.m):
 *   f(R, x) = exp(tr(F^T R)) / c(s) * N(x; mu, Sigma),  F = U diag(s) V^T,
 * c(s) the matrix Fisher normalising constant ('matrix Fisher/pdf_MF_normal.m').
 * U, V: 3x3 row-major; s: 3; mu: ndim; Sigma: row-major 3x3 whose leading
 * ndim x ndim block is used.  The plan's model supplies L.
 * hp_density_mf_gauss writes f (FP64, grid layout f(a,b,c,x...));
 * hp_state_init_mf_gauss loads F = fftSO3R(f) (FP64 transform) into the state
 * without the density leaving the device (HP_REAL plans). */
int hp_density_mf_gauss(hp_plan* plan, const double* U, const double* s, const double* V, const double* mu,
                        const double* Sigma, double* f, int mem);
int hp_state_init_mf_gauss(hp_state* state, const double* U, const double* s, const double* V,
                           const double* mu, const double* Sigma);

/* ---- batches: independent densities advanced together (config 5 of the
 * build's workloads; no counterpart in the reference, whose drivers loop over
 * one density) ----
 * Members are resident states of any plans (bandlimit, omega grid, precision);
 * colls (may be NULL, or NULL entries) makes a member's step the hybrid step.
 * Members on different plans run concurrently on the batch's streams; members
 * sharing a plan share its workspace and run in turn.  hp_batch_step runs one
 * eager warm-up step, then replays a CUDA graph of two batch steps; the graph
 * is rebuilt when dt or method change.  Plan profiling must be off. */
typedef struct hp_batch hp_batch;
int hp_batch_create(hp_state* const* states, hp_collision* const* colls, int n, hp_batch** batch);
int hp_batch_destroy(hp_batch* batch);
int hp_batch_step(hp_batch* batch, double dt, int method, int nsteps);
/* graph replays so far and the number of concurrent streams */
int hp_batch_info(hp_batch* batch, long long* graph_launches, int* concurrent_streams);
/* Persistent plane pass: with enable != 0 the plane passes of the members that
 * take plain Euler steps on 3-D plans (2Bx in 8..32) run as one persistent
 * kernel per round of members, a work queue over (member, tile, k3 plane)
 * items drained by the resident blocks, larger grids first; a round holds at
 * most one member per plan, since members of one plan share its workspace.
 * Hybrid members, other methods and other grids step as before.  The results
 * are those of the per-member passes.  Off by default. */
int hp_batch_set_persistent(hp_batch* batch, int enable);

/* ---- statistics: the raw moments of get_stat (propagation/pendulum.m:547-594,
 * pendulum_reduced_hybrid.m:304-351) ----
 * The moments are computed from the coefficients (F^l_mn with l <= 2 at the
 * omega origin and l <= 1 along the omega axes), which equal the reference's
 * grid sums over f; no pass over the grid density is made.  E[.] denotes
 * c0 sum_grid w_beta (.) f with c0 = (L/2Bx)^n (unnormalised, like get_stat). */
typedef struct {
  double mass;       /* E[1]                                               */
  double ER[9];      /* E[R_kq], index k*3+q                               */
  double ERR[81];    /* E[R_kq R_k'q'], index (k*3+q)*9 + k'*3+q'          */
  double Ex[3];      /* E[x_i] (i < ndim)                                  */
  double Exx[9];     /* E[x_i x_j], index i*3+j (raw, not centred)         */
  double ExR[27];    /* E[x_i R_kq], index i*9 + k*3+q                     */
} hp_moments_t;
/* Moments of the density with coefficients F (full layout).  fx (may be NULL):
 * host buffer of (2Bx)^ndim doubles receiving the R-marginal sum_R w f on the
 * omega grid (first omega index fastest).  Needs B >= 3 and a model (for L). */
int hp_moments(hp_plan* plan, const double* F, int mem, hp_moments_t* out, double* fx);

/* ---- resident state: coefficients kept on the device in the plan's internal
 * layout across steps (the time loops of pendulum.m:269-315 and
 * pendulum_reduced.m:243-289 without host round trips). ---- */
int hp_state_create(hp_plan* plan, hp_state** state);
int hp_state_destroy(hp_state* state);
int hp_state_load(hp_state* state, const double* F, int mem);   /* full layout in  */
int hp_state_store(hp_state* state, double* F, int mem);        /* full layout out */
/* nsteps steps of `method` with step dt.  Mixed-precision 3-D plans keep the
 * coefficients also in FP32 between steps (read by the next step and by
 * hp_state_density); the first call on such a state allocates those two
 * buffers, so make it outside any CUDA stream capture. */
int hp_state_step(hp_state* state, double dt, int method, int nsteps);
/* nsteps hybrid steps of pendulum_reduced_hybrid.m:224-234, each
 *   F = propagate_den(F, f); f = fftSO3R backward(F); f += dt*df(f); F = forward(f)
 * with df the collision operator of `coll` (pendulum_reduced_discrete_propagate,
 * propagation/discrete/mex/sources/pendulum_reduced_collision/propagate.cu:6-121).
 * The plan needs a model: the density-gravity model of hp_plan_set_den_model
 * (the reference's hybrid loop), or a coefficient-gravity model of
 * hp_plan_set_model (then F = propagate(F), e.g. the 3-D pendulum with the
 * 3-D collision operator); coll must be created on the same plan.  The grid
 * density f stays on the device between steps (compute precision). */
int hp_state_hybrid_step(hp_state* state, hp_collision* coll, double dt, int method, int nsteps);
/* Density on the grid of the current state into `f` (device pointer; double
 * for HP_FP64 plans, float for HP_MIXED plans): after hybrid steps the
 * post-collision density f of the last step, otherwise f = ifftSO3R(F). */
int hp_state_density(hp_state* state, void* f);
/* The inverse of hp_state_density: loads F = fftSO3R(f) from a device grid
 * density in the plan's compute precision (fftSO3R_mex('forward',f,d,w),
 * propagation/mex/sources/fftSO3R/kernel.cu:11-195, without host staging). */
int hp_state_load_density(hp_state* state, const void* f);
/* Per-step health check of a resident state (no counterpart in the reference,
 * whose MEX error handlers print and continue, e.g.
 * propagation/mex/sources/pendulum_propagate_reduced_den/setup.cu:7-37).  Every
 * check_every steps of hp_state_step / hp_state_hybrid_step the FP64
 * coefficients are scanned for NaN/Inf (HP_ERR_NONFINITE), and with
 * mass_rtol > 0 the l = 0 mass F^0_00[0] is compared with its value when the
 * guard was set (|m - m0| > mass_rtol |m0|: HP_ERR_MASS_DRIFT).  A failed
 * check ends the call after the failing step, which stays in the state;
 * hp_last_error names the step.  check_every = 0 turns the guard off.  Each
 * check synchronises the plan's stream; inside a stream capture the checks
 * are skipped, and hp_batch_step checks its guarded members after its graph
 * replays.  The first call allocates a 4-byte device flag. */
int hp_state_set_guard(hp_state* state, int check_every, double mass_rtol);
/* Device memory budget of the library (no counterpart in the reference, whose
 * MEX files allocate and free on every call).  hp_set_device_budget caps the
 * device bytes the library holds at once over all devices and objects (plan
 * tables and workspaces, states, collision tables; 0 = no cap); an allocation
 * beyond the cap fails as a failed cudaMalloc does, with HP_ERR_ALLOC.
 * hp_device_bytes returns the bytes held now.  The static scratch array of
 * hp_pendulum_derivative_noalloc is not counted. */
int hp_set_device_budget(long long bytes);
int hp_device_bytes(long long* bytes);
/* F^0_{00}[k=0] (total mass, notes/6 pendulum/pendulum.tex:108-134) of the state. */
int hp_state_mass(hp_state* state, double* mass);
/* hp_moments of the resident state; after hybrid steps these are the moments
 * of the post-collision grid density (its forward transform is the state). */
int hp_state_moments(hp_state* state, hp_moments_t* out, double* fx);
/* l = 0 mass normalisation: scales the state (FP64) so that F^0_{00}[0] == mass;
 * *scale (may be NULL) receives the factor applied.  The derivative conserves
 * F^0_{00}[0] exactly (every term vanishes at l = 0, k = 0), so this only
 * corrects changes made outside the propagation (grid-side collision updates,
 * truncation of a user-supplied density).  No counterpart in the reference. */
int hp_state_normalize(hp_state* state, double mass, double* scale);

#ifdef __cplusplus
}
#endif
#endif /* HP_H */
