/*
 * gpe_b200 -- B200-native backend for GPESolver's solver/ hot path.
 *
 * A C ABI (plain pointers and sizes) that a C++ adapter deriving from the
 * reference's AbstractGrossPitaevskiSolver (src/solver/solver.hpp:17-72) binds
 * one-to-one: every pure virtual of that class has an entry point here, plus
 * fused multi-iteration entry points that run whole reference iterations on the
 * device (CUDA-graph replays, no host round trip per iteration).
 *
 * Conventions kept from the reference:
 *   - grid layout row-major idx = (i*ny + j)*nz + k, x slowest, z fastest
 *     (src/utils/types/mat3d/stdmat3d.hpp:26-28);
 *   - psi on the host is interleaved (re, im) FP64, i.e. std::complex<double>
 *     (src/context/context.hpp:30-36); V and phi are FP64;
 *   - all quantities in atomic units, as PhysicalParameters holds them
 *     (src/parameters/parameters.hpp:10-123).
 *
 * Every call returns 0 on success or a GPE_ERR_* code; gpe_last_error() gives the
 * message of the last failure on the calling thread.  One handle is used by one
 * host thread at a time; distinct handles may be driven from distinct threads.
 */
#ifndef GPE_B200_H
#define GPE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPE_B200_ABI_VERSION 1

enum {
    GPE_OK            = 0,
    GPE_ERR_ARG       = 1, /* invalid argument (null pointer, size mismatch, bad value) */
    GPE_ERR_SIZE      = 2, /* grid size the FFT planner does not support */
    GPE_ERR_CUDA      = 3, /* CUDA runtime error (launch, copy, allocation) */
    GPE_ERR_STATE     = 4, /* call not valid in the handle's current state */
    GPE_ERR_NUMERIC   = 5, /* NaN/Inf detected in a reduction */
    GPE_ERR_NOMEM     = 6  /* device allocation failed */
};

/* Arithmetic of the fields on the device. */
enum {
    GPE_PREC_C64  = 0, /* complex64 psi, FP32 FFT/stencil, FP64 reductions (default) */
    GPE_PREC_C128 = 1  /* complex128 psi, FP64 everywhere (reference precision) */
};

/* The PhysicalParameters fields the solver backend reads
 * (src/parameters/parameters.hpp:10-123), in atomic units. */
typedef struct gpe_params {
    int nx, ny, nz;
    double dx, dy, dz;
    double m;
    double n_atoms;
    double add;            /* dipolar length, 131 a0 (parameters.cpp:43) */
    double cdd;            /* 12 pi add / m */
    double ggp11;          /* 4 pi a / m */
    double gamma;          /* LHY coefficient */
    double w_15;           /* n_atoms^1.5 */
    double real_time_dt;   /* 1.00e10 (parameters.hpp:69-70) */
    double imag_time_dt;   /* 1.25e11 (parameters.hpp:71-72) */
    int const_edd;         /* 1: edd fixed; 0: RT ramps edd_start -> edd_stop */
    double edd, edd_start, edd_stop;
    long iter_real;        /* ramp length (update_edd divides by it) */
    int precision;         /* GPE_PREC_* */
    int device;            /* CUDA device ordinal */
    int schedule;          /* GPE_SCHED_*: kernel schedule of the fused iterations */
} gpe_params;

/* Kernel schedule of gpe_imag_steps / gpe_real_steps. */
enum {
    GPE_SCHED_AUTO  = 0, /* the four-kernel fused pipeline where the grid has compiled
                            line lengths (nx, ny in {32,64,96,128,256}, nz in
                            {8,16,24,32,64}, complex64), else the split schedule */
    GPE_SCHED_SPLIT = 1  /* one kernel per FFT axis pass (any supported grid) */
};

typedef struct gpe_handle gpe_handle;

const char *gpe_last_error(void);
int gpe_abi_version(void);

/* Fill the derived coefficients (add, cdd, ggp11, gamma, w_15) and the default
 * time steps exactly as PhysicalParameters::init_parameters does
 * (src/parameters/parameters.cpp:37-51, parameters.hpp:69-72).  Reads nx..edd. */
int gpe_params_derive(gpe_params *p);

/* Coefficients of PhysicalParameters::update_edd(iter) (parameters.cpp:53-59):
 * out3 = {edd, ggp11, gamma}. */
int gpe_params_edd_at(const gpe_params *p, long iter, double *out3);

/* Lifecycle.  Replaces GpuGrossPitaevskiSolver's constructor, init_containers()
 * and prepare_fft() (src/solver/cuda_solver/gpu_solver.cpp:4-38; solver.hpp:56,66):
 * allocates the device fields, plans the FFTs and builds the dipolar kernel
 * V_dd(k) and the kinetic phase tables in FP64. */
int gpe_create(const gpe_params *p, gpe_handle **out);
int gpe_destroy(gpe_handle *h);

/* Run on a caller-provided cudaStream_t (NULL: the handle's own stream). */
int gpe_set_stream(gpe_handle *h, void *cuda_stream);
int gpe_get_stream(gpe_handle *h, void **cuda_stream);
int gpe_synchronize(gpe_handle *h);

/* --- data in / out (import_data, import_pote, export_data; solver.hpp:68-70) --- */

/* AbstractGrossPitaevskiSolver::load_buffer (solver.cpp:118-125): psi and the
 * scratch copy psii both take the given values, then calc_norm + normalize.
 * n = nx*ny*nz complex values (2n doubles). */
int gpe_load_psi(gpe_handle *h, const double *psi_c128, size_t n);
/* import_data (solver.hpp:69; gpu_solver.cpp:141-148): psi and psii take the given
 * values as they are (no normalisation).  An adapter whose base class runs
 * load_buffer itself calls this, then calc_norm and normalize. */
int gpe_import_psi(gpe_handle *h, const double *psi_c128, size_t n);
/* load_pote (solver.cpp:127-131). n = nx*ny*nz doubles. */
int gpe_load_potential(gpe_handle *h, const double *V, size_t n);
/* export_data: the current psi (normalised if the last step was an imaginary-time
 * step), widened to complex128. */
int gpe_export_psi(gpe_handle *h, double *psi_c128, size_t n);
/* gpe_export_psi without waiting for the copy: psi is widened to complex128 on
 * the device (before any later call's iterations), then copied to psi_c128 on
 * a copy stream of the handle, overlapping the iterations that follow.  Use
 * pinned host memory for the overlap; the buffer must stay valid until
 * gpe_export_wait returns.  A second call waits for the first copy.  (The
 * reference copies psi synchronously at every checkpoint, solver.cpp:54-59,
 * 81-86.) */
int gpe_export_psi_async(gpe_handle *h, double *psi_c128, size_t n);
int gpe_export_wait(gpe_handle *h);
/* The dipolar field fi3d as last computed (FP64 copy). */
int gpe_export_fi3d(gpe_handle *h, double *fi3d, size_t n);
/* Sets the dipolar field fi3d (n = nx*ny*nz doubles).  The reference keeps fi3d
 * in its solver state between real-time iterations: real_time_iter
 * (solver.cpp:107-112) starts with a potential half step that uses the fi3d of
 * the previous iteration's calc_fi3d, which psi alone does not determine.  A run
 * resumed from a checkpoint loads psi and this field to continue exactly where
 * it stopped.  No counterpart in the reference, which has no resume. */
int gpe_load_fi3d(gpe_handle *h, const double *fi3d, size_t n);

/* --- the pure virtuals of AbstractGrossPitaevskiSolver (solver.hpp:55-66) --- */

int gpe_calc_fi3d(gpe_handle *h);                 /* calc_fi3d (Poisson::execute) */
int gpe_imag_iter_linear_step(gpe_handle *h);     /* fused Euler update into psii */
int gpe_imag_iter_nonlinear_step(gpe_handle *h);  /* psi <- psii (nonlinear term is fused above) */
/* xnorma = sum |psi|^2 dV in FP64.  With xnorma == NULL the reduction stays on the
 * device (no host synchronisation); normalize uses the device value either way. */
int gpe_calc_norm(gpe_handle *h, double *xnorma);
int gpe_normalize(gpe_handle *h);                 /* psi /= sqrt(xnorma) */
int gpe_real_fft_potential_half_step(gpe_handle *h);
int gpe_real_fft_kinetic_step(gpe_handle *h);
/* calc_energy: out6 = {e_kin, e_pot, e_int, e_ext (dipolar), e_bmf, e_total}. */
int gpe_calc_energy(gpe_handle *h, double *out6);
/* Coefficients the nonlinear terms use from the next call on (update_edd). */
int gpe_set_coeffs(gpe_handle *h, double ggp11, double gamma);

/* --- fused iterations (the fast path) --- */

/* k reference imaginary-time iterations (imag_time_iter, solver.cpp:99-105). */
int gpe_imag_steps(gpe_handle *h, long k);
/* k reference real-time iterations first_iter .. first_iter+k-1 (real_time_iter,
 * solver.cpp:107-112), applying update_edd(iter) before each one when the
 * handle's const_edd is 0 (calc_evolution, solver.cpp:75-77). */
int gpe_real_steps(gpe_handle *h, long k, long first_iter);

/* `checks` rounds of (k imaginary-time iterations, calc_energy), with the
 * energies kept on the device until the end: e_total[c] = the total energy
 * after round c.  One host synchronisation instead of one per check (the
 * reference's calc_initial_state computes the energy every 100 iterations,
 * solver.cpp:54-59; a convergence loop checks it more often). */
int gpe_imag_steps_energies(gpe_handle *h, long k, int checks, double *e_total);

/* Number of kernels the library launched on this handle since creation. */
int gpe_launch_count(gpe_handle *h, long long *count);

/* Lines per CTA of the fused x pass (kinetic, dipolar pencils: 8 or 16) that
 * the autotuner picked for this grid when the first handle of the grid was
 * created on its device (GPE_X_TILES="k,d" in the environment fixes them);
 * 16, 16 on schedules without the fused x pass.  No reference counterpart (the
 * reference's FFTs are FFTW / cuFFT plans). */
int gpe_x_tiles(gpe_handle *h, int *kin_lines, int *dip_lines);

/* --- measurement --- */

/* Kernels of the real-time iteration, for per-kernel timing. */
enum {
    GPE_K_DIP_Z_FWD = 0, GPE_K_DIP_Y_FWD, GPE_K_DIP_X, GPE_K_DIP_Y_INV, GPE_K_DIP_Z_INV,
    GPE_K_KIN_Z_FWD, GPE_K_KIN_Y_FWD, GPE_K_KIN_X, GPE_K_KIN_Y_INV, GPE_K_KIN_Z_INV,
    GPE_K_PHASE, GPE_K_IT_UPDATE,
    /* the fused pipeline (real time): X pencils, Y inverse, Z rows, Y forward */
    GPE_K_F_X, GPE_K_F_YINV, GPE_K_F_Z, GPE_K_F_YFWD,
    /* kinetic x pencils alone, dipolar x pencils alone, the yz plane kernel
       (grids with a plane kernel: one iteration = F_XK + F_XD + F_YZ) */
    GPE_K_F_XK, GPE_K_F_XD, GPE_K_F_YZ,
    GPE_K_COUNT
};
/* Launches kernel `which` `reps` times back to back on the handle's stream
 * between two CUDA events and reports the mean time per launch and the
 * kernel's algorithmic bytes per launch (compulsory reads + writes of its
 * inputs and outputs).  The solver state is saved before and restored after. */
int gpe_time_kernel(gpe_handle *h, int which, int reps, double *ms_per_launch,
                    double *bytes_per_launch);
/* Name of kernel `which` as it appears in a profiler's launch list. */
const char *gpe_kernel_name(int which);
/* Name of the plane kernel that runs this handle's middle real-time iterations
 * (GPE_K_F_YZ): "k5_yz_pair" (two CTAs per x plane; its imaginary-time
 * counterpart is k5_yz_pair_it) or "k4_yz"; "" on grids without a plane
 * kernel.  No reference counterpart. */
const char *gpe_plane_kernel_name(gpe_handle *h);

/* --- device-side initial state and potential --- */

/* Potential ids, in the reference's registration order
 * (src/parameters/potentials.hpp:76-157). */
enum {
    GPE_POT_HARMONIC = 0, GPE_POT_MEXICAN, GPE_POT_MEXICAN_FREE, GPE_POT_CYLINDRICAL, GPE_POT_FREE,
    GPE_POT_MEXICAN_ASYMETRIC, GPE_POT_MEXICAN_ASYMETRIC_FREE
};
/* Initial-state strategies computed from formulas (InitializationOption,
 * src/parameters/complex_param.hpp:57-97; the file-based ones load psi). */
enum { GPE_INIT_COS = 0, GPE_INIT_GAUSS, GPE_INIT_MULTIPLE_GAUSS, GPE_INIT_SETUP_GAUSS };

/* The PhysicalParameters fields the potentials and initialisers read, in
 * atomic units (parameters.hpp:10-123, as init_parameters leaves them). */
typedef struct gpe_init_params {
    double omega_x, omega_y, omega_z;
    double aa, b;           /* MEXICAN coefficients (parameters.cpp:38-39) */
    double dd;              /* double-well distance */
    int n_gauss_max;        /* MULTIPLE_GAUSS maxima (at most 64) */
    int bec_droplets_x, bec_droplets_y, bec_droplets_z; /* SETUP_GAUSS (product at most 64) */
} gpe_init_params;

/* DataInitializer::init_pote + load_pote (src/initializer/initializer.cpp:229-248,
 * solver.cpp:127-131) computed on the device in FP64: bit-identical to the
 * reference's host potential. */
int gpe_init_potential(gpe_handle *h, int pote, const gpe_init_params *ip);
/* DataInitializer::init_with_* + load_buffer (initializer.cpp:46-219,
 * solver.cpp:118-125) computed on the device in FP64 (exp / cos within an ulp
 * or two of the host library), then normalised as load_buffer does. */
int gpe_init_psi(gpe_handle *h, int strategy, const gpe_init_params *ip);
/* The potential the handle holds (buf_data->pote), widened to FP64. */
int gpe_export_potential(gpe_handle *h, double *V, size_t n);

/* --- batched imaginary time (parameter sweeps) --- */

/* A set of independent solves on one GPU whose imaginary-time iterations run
 * as one CUDA-graph launch per call of up to 1024 iterations (longer calls: one
 * launch per 1024; GPE_BATCH_CHUNK=1..4096 sets the count): every member's
 * kernel chain is an independent branch of the same graph, joined only at its
 * end, so small grids fill the GPU together.  The
 * reference runs such sweeps as separate processes, one after the other.
 * Members may differ in grid and parameters; each must take the fused
 * complex64 pipeline (compiled grid sizes). */
typedef struct gpe_batch gpe_batch;
int gpe_batch_create(const gpe_params *members, int count, gpe_batch **out);
int gpe_batch_destroy(gpe_batch *b);
/* The handle of member m (owned by the batch): load, initialise, export and
 * measure members with the single-handle calls. */
int gpe_batch_member(gpe_batch *b, int m, gpe_handle **h);
/* Stream of the batch and of every member (NULL: the batch's own stream). */
int gpe_batch_set_stream(gpe_batch *b, void *cuda_stream);
/* k imaginary-time iterations of every member (gpe_imag_steps on each). */
int gpe_batch_imag_steps(gpe_batch *b, long k);

/* --- learned warm start for imaginary time (no counterpart in the reference) --- */

/* A network maps the physical parameters of a solve (normalised inputs, e.g.
 * edd, n_atoms, omega_r, omega_z) to an amplitude |psi_0| on the solver grid;
 * imaginary time refines it instead of starting from an initialiser.
 *   dense n_inputs -> hidden, SiLU; dense hidden -> channels[0] x latent
 *   volume (grid / 2^levels), SiLU; `levels` x (nearest x2 upsampling, 3x3x3
 *   convolution channels[s] -> channels[s+1], SiLU); 3x3x3 convolution
 *   channels[levels] -> 1 (the amplitude, linear).
 * Weights BF16, arithmetic FP32; training: mean squared amplitude error, Adam
 * on FP32 master weights.  Channel counts: 1, 2, 4, 8, 16 or 32. */
typedef struct gpe_warm_config {
    int nx, ny, nz;      /* output grid, divisible by 2^levels */
    int levels;          /* upsampling convolution stages (0..6) */
    int channels[8];     /* channels[0..levels] */
    int hidden;          /* width of the first dense layer */
    int n_inputs;        /* scalar inputs per solve */
    int max_batch;       /* largest batch of forward / training calls */
} gpe_warm_config;
typedef struct gpe_warm gpe_warm;
int gpe_warm_create(const gpe_warm_config *cfg, int device, gpe_warm **out);
int gpe_warm_destroy(gpe_warm *w);
/* number of FP32 weights (the flat layout set / get use) */
int gpe_warm_num_weights(gpe_warm *w, size_t *n);
int gpe_warm_set_weights(gpe_warm *w, const float *host, size_t n);
int gpe_warm_get_weights(gpe_warm *w, float *host, size_t n);
/* fan-in-scaled uniform initialisation from a seed (host generator) */
int gpe_warm_init_weights(gpe_warm *w, unsigned long long seed);
/* amplitudes of B solves (inputs B x n_inputs on the host) into amp_dev
 * (device, B x nx*ny*nz floats) */
int gpe_warm_forward(gpe_warm *w, const float *inputs, int B, float *amp_dev);
/* loss and gradient (host, num_weights floats; NULL: kept on the device) of
 * the mean squared error against targets_dev (device, B x nx*ny*nz) */
int gpe_warm_gradients(gpe_warm *w, const float *inputs, const float *targets_dev, int B, float *grad,
                       double *loss);
/* one Adam step on a batch */
int gpe_warm_train_step(gpe_warm *w, const float *inputs, const float *targets_dev, int B, float lr,
                        double *loss);

/* Amplitude |psi| of the handle's (normalised) psi into a device buffer (FP32),
 * and load_buffer of a real amplitude given on the device (FP32): the hand-off
 * between a solver and the warm-start network without a host round trip.  The
 * loaded state is max(amp, 0) on the interior and zero on the boundary cells,
 * as the reference's initialisers leave them (initializer.cpp:46-219);
 * imaginary time never updates the boundary. */
int gpe_export_amplitude_device(gpe_handle *h, float *amp_dev, size_t n);
int gpe_load_amplitude_device(gpe_handle *h, const float *amp_dev, size_t n);

/* --- allocation-free variant --- */

/* Size of the file-scope device array gpe_calc_fi3d_noalloc works in. */
#define GPE_NOALLOC_SCRATCH_BYTES (16u << 20)

/* calc_fi3d for callers that cannot allocate device memory (a framework that
 * owns all device memory through its own allocator, or a loop that must not
 * add the device-wide synchronisation cudaMalloc/cudaFree can cause).  This
 * entry point has no counterpart in the reference.  It computes the dipolar
 * field phi of a complex64 psi already on the device, with the same kernels as
 * gpe_calc_fi3d, and allocates nothing: its intermediates live in one
 * file-scope __device__ array of GPE_NOALLOC_SCRATCH_BYTES (16 MiB) that every
 * GPU loading the library keeps until the process exits.
 *   psi_c64_dev  device pointer, nx*ny*nz interleaved (re, im) floats, normalised psi
 *   fi3d_dev     device pointer, nx*ny*nz floats (output)
 *   n_atoms      w in rho = w |psi|^2
 *   cuda_stream  cudaStream_t to launch on (NULL: the legacy default stream)
 * Grids whose scratch exceeds the limit are rejected with GPE_ERR_SIZE
 * (128 x 128 x 32 needs about 10.9 MB).  All calls on a GPU share the array, so
 * calls that overlap on one GPU race; each call rebuilds the tables it needs,
 * so nothing carries over from one call to the next.  The first call on each device does a
 * one-time host-side set-up (device address of the array, kernel attributes);
 * make it before any stream capture on that device. */
int gpe_calc_fi3d_noalloc(const void *psi_c64_dev, float *fi3d_dev, int nx, int ny, int nz,
                          double dx, double dy, double dz, double n_atoms, void *cuda_stream);

#ifdef __cplusplus
}
#endif

#endif
