/*
 * CPU FP64 restatement of GPESolver's solver hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This is the oracle the CUDA path is checked against.  It restates, in plain C,
 * the reference's CPU backend (src/solver/cpu_solver/cpu_solver.cpp), its FFTW
 * solvers (src/solver/fft_solvers/cpu/*.cpp), the coefficient derivation
 * (src/parameters/parameters.cpp:37-59), the grid (src/context/context.cpp:17-34),
 * the potentials (src/parameters/potentials.hpp:76-157) and the initialisers
 * (src/initializer/initializer.cpp:46-219), operation for operation, so that with
 * the same FFT it reproduces the compiled reference bit for bit (pinned by
 * tests/test_oracle_pin.py against oracle/_ref/libgpe_ref.so and the golden
 * vectors in tests/golden/).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline may load it.
 */
#ifndef GPE_ORACLE_H
#define GPE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Physical parameters in atomic units, mirroring PhysicalParameters
 * (src/parameters/parameters.hpp:10-123). */
typedef struct {
    int nx, ny, nz;
    double dx, dy, dz;
    double m;
    double n_atoms;
    double omega_x, omega_y, omega_z;
    double dd;
    int const_edd;
    double edd, edd_start, edd_stop;
    long iter_imag, iter_real;
    double real_time_dt; /* 1.00e10 (parameters.hpp:69-70) */
    double imag_time_dt; /* 1.25e11 (parameters.hpp:71-72) */
    int fftw_n_threads;
    /* derived by gpeo_init_parameters */
    double aa, b, dxdydz, add, cdd, ggp11, gamma, w_15;
} gpeo_params;

/* UnitConverter (src/utils/units/units.cpp:3-41). */
double gpeo_len_nm_to_au(double nm);
double gpeo_len_au_to_nm(double au);
double gpeo_mass_da_to_au(double da);
double gpeo_freq_hz_to_au(double hz);
double gpeo_ene_au_to_mev(double au);

void gpeo_default_dt(gpeo_params *p);
void gpeo_init_parameters(gpeo_params *p);
void gpeo_update_edd(gpeo_params *p, unsigned iter);

/* Potential ids follow the reference's registration order
 * (src/parameters/potentials.hpp:76-157). */
enum {
    GPEO_HARMONIC = 0,
    GPEO_MEXICAN,
    GPEO_MEXICAN_FREE,
    GPEO_CYLINDRICAL,
    GPEO_FREE,
    GPEO_MEXICAN_ASYMETRIC,
    GPEO_MEXICAN_ASYMETRIC_FREE
};
/* Initialisers (InitializationOption, src/parameters/complex_param.hpp:57-97). */
enum { GPEO_INIT_COS = 0, GPEO_INIT_GAUSS, GPEO_INIT_MULTIPLE_GAUSS, GPEO_INIT_SETUP_GAUSS };

void gpeo_coords(const gpeo_params *p, double *x, double *y, double *z);
int gpeo_potential(const gpeo_params *p, int pote_id, double *V);
int gpeo_init_psi(const gpeo_params *p, int strategy, int n_gauss_max, int bdx, int bdy, int bdz,
                  double *psi_c128);

typedef struct gpeo_solver gpeo_solver;

gpeo_solver *gpeo_create(const gpeo_params *p);
void gpeo_destroy(gpeo_solver *s);
gpeo_params *gpeo_solver_params(gpeo_solver *s);

/* Field access (row-major (i*ny + j)*nz + k; psi interleaved re, im). */
double *gpeo_psi(gpeo_solver *s);
double *gpeo_psii(gpeo_solver *s);
double *gpeo_fi3d(gpeo_solver *s);
double *gpeo_pote(gpeo_solver *s);

/* AbstractGrossPitaevskiSolver::load_buffer / load_pote (src/solver/solver.cpp:118-131). */
void gpeo_load_buffer(gpeo_solver *s, const double *psi_c128);
void gpeo_load_pote(gpeo_solver *s, const double *V);

/* The virtuals of CpuGrossPitaevskiSolver. */
void gpeo_calc_fi3d(gpeo_solver *s);
void gpeo_imag_iter_linear_step(gpeo_solver *s);
void gpeo_imag_iter_nonlinear_step(gpeo_solver *s);
double gpeo_calc_norm(gpeo_solver *s);
void gpeo_normalize(gpeo_solver *s);
void gpeo_real_fft_potential_half_step(gpeo_solver *s);
void gpeo_real_fft_kinetic_step(gpeo_solver *s);
void gpeo_calc_energy(gpeo_solver *s, double out6[6]);

/* imag_time_iter / real_time_iter (src/solver/solver.cpp:99-112). */
void gpeo_imag_time_iter(gpeo_solver *s);
void gpeo_real_time_iter(gpeo_solver *s);
/* k iterations; RT applies the edd ramp before each iteration
 * (src/solver/solver.cpp:72-77). */
void gpeo_imag_steps(gpeo_solver *s, long k);
void gpeo_real_steps(gpeo_solver *s, long k, long first_iter);

#ifdef __cplusplus
}
#endif

#endif
