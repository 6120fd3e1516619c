/*
 * CPU FP64 restatement of GPESolver's solver hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Each function cites the reference file:line it restates.  The order of every
 * floating-point operation follows the reference's C++ expressions (including
 * std::pow / std::abs, which libstdc++ lowers to pow() and hypot()), so that the
 * same FFT gives the same bits.  FFTs go through the FFTW-API shim in
 * oracle/fftw_shim, exactly as the reference's FFTW solvers call FFTW.
 */
#define _GNU_SOURCE
#include "gpe_oracle.h"

#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------------
 * Units: src/utils/units/units.cpp:3-41
 * ------------------------------------------------------------------------ */
double gpeo_len_nm_to_au(double nm) { return nm * 18.897261260649092; }
double gpeo_len_au_to_nm(double au) { return au * 0.05291772105; }
double gpeo_mass_da_to_au(double da) { return da / 0.000548579909; }
double gpeo_freq_hz_to_au(double hz) { return hz * (4.1356e-12 / 27211.6); }
double gpeo_ene_au_to_mev(double au) { return au * 27211.407953; }

/* Compile-time time steps: src/parameters/parameters.hpp:69-72. */
void gpeo_default_dt(gpeo_params *p) {
    p->real_time_dt = 1.00e10;
    p->imag_time_dt = 1.25e11;
}

/* PhysicalParameters::init_parameters: src/parameters/parameters.cpp:37-51. */
void gpeo_init_parameters(gpeo_params *p) {
    p->aa     = p->m * pow(p->omega_x, 2) / 4. / pow(p->dd, 2);
    p->b      = 0.5 * p->m * pow(p->omega_x, 2);
    p->dxdydz = p->dx * p->dy * p->dz;
    p->add    = 131.;
    p->cdd    = 12. * M_PI * p->add / p->m;
    double a  = p->add / p->edd;
    p->ggp11  = 4. * M_PI * a / p->m;
    p->gamma  = 128. * sqrt(M_PI) * pow(a, 2.5) / 3. / p->m * (1. + 1.5 * pow(p->edd, 2));
    p->w_15   = pow(p->n_atoms, 1.5);
}

/* PhysicalParameters::update_edd: src/parameters/parameters.cpp:53-59. */
void gpeo_update_edd(gpeo_params *p, unsigned iter) {
    p->edd   = p->edd_start + (p->edd_stop - p->edd_start) * iter / (double)(size_t)p->iter_real;
    double a = p->add / p->edd;
    p->ggp11 = 4 * M_PI * a / p->m;
    p->gamma = 128. * sqrt(M_PI) * pow(a, 2.5) / 3. / p->m * (1. + 1.5 * pow(p->edd, 2));
}

/* SimulationContext::initialize: src/context/context.cpp:17-34. */
void gpeo_coords(const gpeo_params *p, double *x, double *y, double *z) {
    for (int i = 0; i < p->nx; i++)
        x[i] = (i - (int)(p->nx / 2)) * p->dx;
    for (int j = 0; j < p->ny; j++)
        y[j] = (j - (int)(p->ny / 2)) * p->dy;
    for (int k = 0; k < p->nz; k++)
        z[k] = (k - (int)(p->nz / 2)) * p->dz;
}

/* PotentialRegistry entries: src/parameters/potentials.hpp:76-157. */
static double pote_eval(const gpeo_params *p, int id, double x, double y, double z) {
    switch (id) {
    case GPEO_HARMONIC: {
        double vx = 0.5 * p->m * pow(x, 2) * pow(p->omega_x, 2);
        double vy = 0.5 * p->m * pow(y, 2) * pow(p->omega_y, 2);
        double vz = 0.5 * p->m * pow(z, 2) * pow(p->omega_z, 2);
        return vx + vy + vz;
    }
    case GPEO_MEXICAN: {
        double vx = -p->b * pow(x, 2) + p->aa * pow(x, 4);
        double vy = 0.5 * p->m * pow(y, 2) * pow(p->omega_y, 2);
        double vz = 0.5 * p->m * pow(z, 2) * pow(p->omega_z, 2);
        return vx + vy + vz;
    }
    case GPEO_MEXICAN_FREE: {
        double vx = p->aa * pow(x, 4);
        double vy = 0.5 * p->m * pow(y, 2) * pow(p->omega_y, 2);
        double vz = 0.5 * p->m * pow(z, 2) * pow(p->omega_z, 2);
        return vx + vy + vz;
    }
    case GPEO_CYLINDRICAL: {
        double r  = sqrt(x * x + y * y);
        double vr = 0.5 * p->m * pow(r, 2) * pow((p->omega_y + p->omega_x) / 2., 2);
        double vz = 0.5 * p->m * pow(z, 2) * pow(p->omega_z, 2);
        return vr + vz;
    }
    case GPEO_FREE: {
        double vz = 0.5 * p->m * pow(z, 2) * pow(p->omega_z, 2);
        return vz;
    }
    case GPEO_MEXICAN_ASYMETRIC: {
        double conv  = 27211.4 * 11.6 * 1e9;
        double nK25  = 0.25 / conv;
        double slope = nK25 / p->dd;
        double vx    = -p->b * pow(x, 2) + p->aa * pow(x, 4) - slope * x;
        double vy    = 0.5 * p->m * pow(y, 2) * pow(p->omega_y, 2);
        double vz    = 0.5 * p->m * pow(z, 2) * pow(p->omega_z, 2);
        return vx + vy + vz;
    }
    case GPEO_MEXICAN_ASYMETRIC_FREE: {
        double conv  = 27211.4 * 11.6 * 1e9;
        double nK25  = 0.25 / conv;
        double slope = nK25 / p->dd;
        double vx    = p->aa * pow(x, 4) - slope * x;
        double vy    = 0.5 * p->m * pow(y, 2) * pow(p->omega_y, 2);
        double vz    = 0.5 * p->m * pow(z, 2) * pow(p->omega_z, 2);
        return vx + vy + vz;
    }
    default:
        return NAN;
    }
}

/* DataInitializer::init_pote: src/initializer/initializer.cpp:229-248.
 * The initializer keeps the registry's function in a
 * std::function<double(int, int, int)> (src/initializer/initializer.hpp:37), so
 * each coordinate (in bohr) is truncated toward zero to an int before the
 * potential is evaluated.  That truncation is reproduced here. */
int gpeo_potential(const gpeo_params *p, int id, double *V) {
    if (id < GPEO_HARMONIC || id > GPEO_MEXICAN_ASYMETRIC_FREE)
        return 1;
    double *x = malloc(sizeof(double) * p->nx), *y = malloc(sizeof(double) * p->ny),
           *z = malloc(sizeof(double) * p->nz);
    gpeo_coords(p, x, y, z);
    for (int i = 0; i < p->nx; i++)
        for (int j = 0; j < p->ny; j++)
            for (int k = 0; k < p->nz; k++)
                V[((size_t)i * p->ny + j) * p->nz + k] =
                    pote_eval(p, id, (double)(int)x[i], (double)(int)y[j], (double)(int)z[k]);
    free(x);
    free(y);
    free(z);
    return 0;
}

/* DataInitializer::init_with_* : src/initializer/initializer.cpp:46-219.  Only
 * the interior 1..n-2 is written; the boundary stays zero. */
int gpeo_init_psi(const gpeo_params *p, int strategy, int n_gauss_max, int bdx, int bdy, int bdz,
                  double *psi) {
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    memset(psi, 0, sizeof(double) * 2 * (size_t)nx * ny * nz);
    double *x = malloc(sizeof(double) * nx), *y = malloc(sizeof(double) * ny),
           *z = malloc(sizeof(double) * nz);
    gpeo_coords(p, x, y, z);
    int rc = 0;

    double *cx = NULL, *cy = NULL, *cz = NULL;
    int nmax = 0;
    if (strategy == GPEO_INIT_MULTIPLE_GAUSS) {
        /* init_with_multiple_gaussian: :162-219 */
        nmax = n_gauss_max;
        cx   = calloc(nmax > 0 ? nmax : 1, sizeof(double));
        cy   = calloc(nmax > 0 ? nmax : 1, sizeof(double));
        for (int idx = 0; idx < nmax; idx++) {
            cx[idx] = idx % 2 ? p->dd : -p->dd;
            if (nmax % 2 == 1) {
                int center_y_idx = nmax / 2;
                double y_offset  = (idx - center_y_idx) * (p->ny * p->dy) / 2. / (nmax + 1.);
                cy[idx]          = y_offset;
            }
            if (nmax % 2 == 0) {
                int y_idx       = (idx / 2 + 1);
                int y_maximas   = (nmax / 2 + 1);
                double y_offset = y_idx * (p->ny * p->dy) / y_maximas;
                cy[idx]         = y[0] + y_offset;
            }
        }
    } else if (strategy == GPEO_INIT_SETUP_GAUSS) {
        /* init_with_setup_gaussian: :101-160 */
        nmax         = bdx * bdy * bdz;
        cx           = calloc(nmax > 0 ? nmax : 1, sizeof(double));
        cy           = calloc(nmax > 0 ? nmax : 1, sizeof(double));
        cz           = calloc(nmax > 0 ? nmax : 1, sizeof(double));
        double x_tot = p->nx * p->dx;
        double y_tot = p->ny * p->dy;
        double z_tot = p->nz * p->dz;
        for (int i = 0; i < bdx; i++)
            for (int j = 0; j < bdy; j++)
                for (int k = 0; k < bdz; k++) {
                    int idx          = i * bdy * bdz + j * bdz + k;
                    double spacing_x = x_tot / (double)(bdx + 1);
                    double spacing_y = y_tot / (double)(bdy + 1);
                    double spacing_z = z_tot / (double)(bdz + 1);
                    cx[idx]          = -x_tot / 2 + spacing_x * (i + 1);
                    cy[idx]          = -y_tot / 2 + spacing_y * (j + 1);
                    cz[idx]          = -z_tot / 2 + spacing_z * (k + 1);
                }
    } else if (strategy != GPEO_INIT_COS && strategy != GPEO_INIT_GAUSS) {
        rc = 1;
    }

    for (int i = 1; i < nx - 1 && rc == 0; i++) {
        for (int j = 1; j < ny - 1; j++) {
            for (int k = 1; k < nz - 1; k++) {
                double val = 0.0;
                if (strategy == GPEO_INIT_COS) {
                    /* init_with_cos: :46-71 */
                    double xx     = x[i] - p->dd;
                    double yy     = y[j];
                    double zz     = z[k];
                    double rrr    = ((int)(p->nx / 2) * p->dx);
                    double cos_x  = cos(2 * M_PI * xx / rrr);
                    double cos_y  = cos(2 * M_PI * yy / rrr);
                    double cos_z  = cos(1 * M_PI * zz / rrr);
                    val           = cos_x * cos_y * cos_z;
                } else if (strategy == GPEO_INIT_GAUSS) {
                    /* init_with_gaussian: :73-99 */
                    double xx      = x[i], yy = y[j], zz = z[k];
                    double sigma_x = (p->nx * p->dx) / 10.;
                    double sigma_y = (p->ny * p->dy) / 10.;
                    double sigma_z = (p->nz * p->dz) / 10.;
                    val            = exp(-0.5 * (xx * xx) / (sigma_x * sigma_x)) *
                          exp(-0.5 * (yy * yy) / (sigma_y * sigma_y)) *
                          exp(-0.5 * (zz * zz) / (sigma_z * sigma_z));
                } else {
                    double xx      = x[i], yy = y[j], zz = z[k];
                    double sigma_x = (p->nx * p->dx) / 20.;
                    double sigma_y = (p->ny * p->dy) / 20.;
                    double sigma_z = (p->nz * p->dz) / 20.;
                    val            = 0.0;
                    for (int m = 0; m < nmax; m++) {
                        double xc = xx - cx[m];
                        double yc = yy - cy[m];
                        double zc = (strategy == GPEO_INIT_SETUP_GAUSS) ? zz - cz[m] : zz;
                        val += exp(-0.5 * (xc * xc) / (sigma_x * sigma_x)) *
                               exp(-0.5 * (yc * yc) / (sigma_y * sigma_y)) *
                               exp(-0.5 * (zc * zc) / (sigma_z * sigma_z));
                    }
                }
                size_t idx       = ((size_t)i * ny + j) * nz + k;
                psi[2 * idx]     = val;
                psi[2 * idx + 1] = 0.0;
            }
        }
    }
    free(cx);
    free(cy);
    free(cz);
    free(x);
    free(y);
    free(z);
    return rc;
}

/* ---------------------------------------------------------------------------
 * Solver state: CPUSolverData (src/solver/solver_data/cpu_solver_data.hpp:11-32)
 * plus the two FFTW solvers' buffers and tables.
 * ------------------------------------------------------------------------ */
struct gpeo_solver {
    gpeo_params p;
    double *cpsi, *cpsii, *fi3d, *pote; /* N complex / N complex / N / N */
    double xnorma;
    /* FFTWPoissonSolver */
    double *rho_r;  /* 8N reals */
    double *rho_k;  /* 2nx*2ny*(nz+1) complex */
    double *vdip_k; /* same, complex (imag always 0) */
    fftw_plan pois_fwd, pois_bwd;
    /* FFTWRealTimeSplitSolver */
    double *sp_r, *sp_k; /* N complex each */
    double *kin;         /* N reals */
    fftw_plan sp_fwd, sp_bwd;
};

#define IDX(s, i, j, k) ((((size_t)(i)) * (s)->p.ny + (j)) * (s)->p.nz + (k))

gpeo_params *gpeo_solver_params(gpeo_solver *s) { return &s->p; }
double *gpeo_psi(gpeo_solver *s) { return s->cpsi; }
double *gpeo_psii(gpeo_solver *s) { return s->cpsii; }
double *gpeo_fi3d(gpeo_solver *s) { return s->fi3d; }
double *gpeo_pote(gpeo_solver *s) { return s->pote; }

/* FFTWPoissonSolver::prepare_containers: fftw_poisson_solver.cpp:12-49. */
static void poisson_prepare(gpeo_solver *s) {
    const int nx = 2 * s->p.nx, ny = 2 * s->p.ny, nz = 2 * s->p.nz;
    const double dx = s->p.dx, dy = s->p.dy, dz = s->p.dz;
    const double dkx = 2. * M_PI / (nx * dx);
    const double dky = 2. * M_PI / (ny * dy);
    const double dkz = 2. * M_PI / (nz * dz);
    for (int i = 0; i < nx; ++i) {
        double kx = (i <= (nx / 2)) ? i * dkx : (i - nx) * dkx;
        for (int j = 0; j < ny; ++j) {
            double ky = (j <= (ny / 2)) ? j * dky : (j - ny) * dky;
            for (int k = 0; k < nz / 2 + 1; ++k) {
                size_t idx = ((size_t)i * ny + j) * (nz / 2 + 1) + k;
                double kz  = (k <= (nz / 2)) ? k * dkz : (k - nz) * dkz;
                double k2  = kx * kx + ky * ky + kz * kz;
                if (k2 > 1e-30) {
                    s->vdip_k[2 * idx]     = (kz * kz / k2);
                    s->vdip_k[2 * idx + 1] = 0.0;
                } else {
                    s->vdip_k[2 * idx]     = 0.0;
                    s->vdip_k[2 * idx + 1] = 0.0;
                }
            }
        }
    }
}

/* FFTWRealTimeSplitSolver::prepare_containers: fftw_split_solver.cpp:11-42. */
static void split_prepare(gpeo_solver *s) {
    const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
    const double dx = s->p.dx, dy = s->p.dy, dz = s->p.dz;
    const double dt = s->p.real_time_dt;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                double kx = (i <= nx / 2) ? (2.0 * M_PI * i / (nx * dx))
                                          : (2.0 * M_PI * (i - nx) / (nx * dx));
                double ky = (j <= ny / 2) ? (2.0 * M_PI * j / (ny * dy))
                                          : (2.0 * M_PI * (j - ny) / (ny * dy));
                double kz = (k <= nz / 2) ? (2.0 * M_PI * k / (nz * dz))
                                          : (2.0 * M_PI * (k - nz) / (nz * dz));
                double k_sq                        = kx * kx + ky * ky + kz * kz;
                double factor                      = -dt / (2.0 * s->p.m) * k_sq;
                s->kin[(size_t)i * ny * nz + j * nz + k] = factor;
            }
}

/* AbstractGrossPitaevskiSolver::initialize (src/solver/solver.cpp:15-23):
 * allocate (zeroed, stdmat3d.hpp:87), plan both FFT solvers (fft_context.cpp:30-42),
 * then calc_norm + normalize on the zero psi (which divides 0 by 0: the reference
 * leaves NaN-free zeros only because the buffers are overwritten by load_buffer). */
gpeo_solver *gpeo_create(const gpeo_params *p) {
    gpeo_solver *s = calloc(1, sizeof(*s));
    s->p           = *p;
    const size_t N = (size_t)p->nx * p->ny * p->nz;
    s->cpsi        = calloc(2 * N, sizeof(double));
    s->cpsii       = calloc(2 * N, sizeof(double));
    s->fi3d        = calloc(N, sizeof(double));
    s->pote        = calloc(N, sizeof(double));

    const int px = 2 * p->nx, py = 2 * p->ny, pz = 2 * p->nz;
    const size_t NP = (size_t)px * py * pz, NPo = (size_t)px * py * (pz / 2 + 1);
    s->rho_r        = fftw_malloc(sizeof(double) * NP);
    s->rho_k        = fftw_malloc(sizeof(double) * 2 * NPo);
    s->vdip_k       = malloc(sizeof(double) * 2 * NPo);
    int nth         = p->fftw_n_threads > 0 ? p->fftw_n_threads : 4;
    fftw_plan_with_nthreads(nth);
    s->pois_fwd = fftw_plan_dft_r2c_3d(px, py, pz, s->rho_r, (fftw_complex *)s->rho_k, FFTW_MEASURE);
    fftw_plan_with_nthreads(nth);
    s->pois_bwd = fftw_plan_dft_c2r_3d(px, py, pz, (fftw_complex *)s->rho_k, s->rho_r, FFTW_MEASURE);
    poisson_prepare(s);

    s->sp_r = fftw_malloc(sizeof(double) * 2 * N);
    s->sp_k = fftw_malloc(sizeof(double) * 2 * N);
    s->kin  = malloc(sizeof(double) * N);
    fftw_plan_with_nthreads(nth);
    s->sp_fwd = fftw_plan_dft_3d(p->nx, p->ny, p->nz, (fftw_complex *)s->sp_r,
                                 (fftw_complex *)s->sp_k, FFTW_FORWARD, FFTW_MEASURE);
    fftw_plan_with_nthreads(nth);
    s->sp_bwd = fftw_plan_dft_3d(p->nx, p->ny, p->nz, (fftw_complex *)s->sp_k,
                                 (fftw_complex *)s->sp_r, FFTW_BACKWARD, FFTW_MEASURE);
    split_prepare(s);
    return s;
}

void gpeo_destroy(gpeo_solver *s) {
    if (!s)
        return;
    fftw_destroy_plan(s->pois_fwd);
    fftw_destroy_plan(s->pois_bwd);
    fftw_destroy_plan(s->sp_fwd);
    fftw_destroy_plan(s->sp_bwd);
    fftw_free(s->rho_r);
    fftw_free(s->rho_k);
    free(s->vdip_k);
    fftw_free(s->sp_r);
    fftw_free(s->sp_k);
    free(s->kin);
    free(s->cpsi);
    free(s->cpsii);
    free(s->fi3d);
    free(s->pote);
    free(s);
}

/* CpuGrossPitaevskiSolver::calc_norm: cpu_solver.cpp:19-34. */
double gpeo_calc_norm(gpeo_solver *s) {
    const size_t N = (size_t)s->p.nx * s->p.ny * s->p.nz;
    double x       = 0.0;
    for (size_t t = 0; t < N; ++t)
        x += s->cpsi[2 * t] * s->cpsi[2 * t] + s->cpsi[2 * t + 1] * s->cpsi[2 * t + 1];
    x *= s->p.dxdydz;
    s->xnorma = x;
    return x;
}

/* CpuGrossPitaevskiSolver::normalize: cpu_solver.cpp:36-48. */
void gpeo_normalize(gpeo_solver *s) {
    const size_t N = (size_t)s->p.nx * s->p.ny * s->p.nz;
    for (size_t t = 0; t < N; ++t) {
        s->cpsi[2 * t] /= sqrt(s->xnorma);
        s->cpsi[2 * t + 1] /= sqrt(s->xnorma);
    }
}

/* AbstractGrossPitaevskiSolver::load_buffer: solver.cpp:118-125. */
void gpeo_load_buffer(gpeo_solver *s, const double *psi) {
    const size_t N = (size_t)s->p.nx * s->p.ny * s->p.nz;
    memcpy(s->cpsi, psi, sizeof(double) * 2 * N);
    memcpy(s->cpsii, psi, sizeof(double) * 2 * N);
    gpeo_calc_norm(s);
    gpeo_normalize(s);
}

/* AbstractGrossPitaevskiSolver::load_pote: solver.cpp:127-131. */
void gpeo_load_pote(gpeo_solver *s, const double *V) {
    const size_t N = (size_t)s->p.nx * s->p.ny * s->p.nz;
    memcpy(s->pote, V, sizeof(double) * N);
}

/* FFTWPoissonSolver::execute: fftw_poisson_solver.cpp:51-96. */
void gpeo_calc_fi3d(gpeo_solver *s) {
    const int nx = 2 * s->p.nx, ny = 2 * s->p.ny, nz = 2 * s->p.nz;
    const size_t N = (size_t)nx * ny * nz, N_out = (size_t)nx * ny * (nz / 2 + 1);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                size_t idx = ((size_t)i * ny + j) * nz + k;
                if (i < nx / 2 && j < ny / 2 && k < nz / 2) {
                    size_t q     = IDX(s, i, j, k);
                    double re    = s->cpsi[2 * q], im = s->cpsi[2 * q + 1];
                    s->rho_r[idx] = (re * re + im * im) * s->p.n_atoms;
                } else {
                    s->rho_r[idx] = 0;
                }
            }
    fftw_execute(s->pois_fwd);
    for (size_t idx = 0; idx < N_out; ++idx) {
        double ar = s->rho_k[2 * idx], ai = s->rho_k[2 * idx + 1];
        double br = s->vdip_k[2 * idx], bi = s->vdip_k[2 * idx + 1];
        s->rho_k[2 * idx]     = ar * br - ai * bi;
        s->rho_k[2 * idx + 1] = ar * bi + ai * br;
    }
    fftw_execute(s->pois_bwd);
    const double norm_factor = 1.0 / (double)N;
    for (int i = 0; i < nx / 2; i++)
        for (int j = 0; j < ny / 2; j++)
            for (int k = 0; k < nz / 2; k++) {
                size_t idx            = ((size_t)i * ny + j) * nz + k;
                s->fi3d[IDX(s, i, j, k)] = s->rho_r[idx] * norm_factor;
            }
}

/* CpuGrossPitaevskiSolver::imag_iter_linear_step: cpu_solver.cpp:50-73. */
void gpeo_imag_iter_linear_step(gpeo_solver *s) {
    const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
    const double *c = s->cpsi;
    double *o       = s->cpsii;
    const double m = s->p.m, dt = s->p.imag_time_dt, cdd = s->p.cdd;
    for (int i = 1; i < nx - 1; i++)
        for (int j = 1; j < ny - 1; j++)
            for (int k = 1; k < nz - 1; k++) {
                size_t q = IDX(s, i, j, k);
                size_t xm = IDX(s, i - 1, j, k), xp = IDX(s, i + 1, j, k);
                size_t ym = IDX(s, i, j - 1, k), yp = IDX(s, i, j + 1, k);
                size_t zm = IDX(s, i, j, k - 1), zp = IDX(s, i, j, k + 1);
                double v  = s->pote[q];
                double cx = -0.5 / (m * pow(s->p.dx, 2));
                double cy = 0.5 / (m * pow(s->p.dy, 2));
                double cz = 0.5 / (m * pow(s->p.dz, 2));
                double c1r, c1i;
                {
                    double Xr = (c[2 * xm] + c[2 * xp]) - 2. * c[2 * q];
                    double Xi = (c[2 * xm + 1] + c[2 * xp + 1]) - 2. * c[2 * q + 1];
                    double Yr = (c[2 * ym] + c[2 * yp]) - 2. * c[2 * q];
                    double Yi = (c[2 * ym + 1] + c[2 * yp + 1]) - 2. * c[2 * q + 1];
                    double Zr = (c[2 * zm] + c[2 * zp]) - 2. * c[2 * q];
                    double Zi = (c[2 * zm + 1] + c[2 * zp + 1]) - 2. * c[2 * q + 1];
                    double vv = v + cdd * s->fi3d[q];
                    c1r       = ((cx * Xr - cy * Yr) - cz * Zr) + c[2 * q] * vv;
                    c1i       = ((cx * Xi - cy * Yi) - cz * Zi) + c[2 * q + 1] * vv;
                }
                o[2 * q]     = c[2 * q] - dt * c1r;
                o[2 * q + 1] = c[2 * q + 1] - dt * c1i;
            }
}

/* CpuGrossPitaevskiSolver::imag_iter_nonlinear_step: cpu_solver.cpp:75-97. */
void gpeo_imag_iter_nonlinear_step(gpeo_solver *s) {
    const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
    const double *c = s->cpsi;
    double *o       = s->cpsii;
    const double w  = s->p.n_atoms;
    for (int i = 1; i < nx - 1; i++)
        for (int j = 1; j < ny - 1; j++)
            for (int k = 1; k < nz - 1; k++) {
                size_t q   = IDX(s, i, j, k);
                double re  = c[2 * q], im = c[2 * q + 1];
                double nrm = re * re + im * im;
                double g3  = (s->p.ggp11 - s->p.cdd / 3) * nrm;
                double gm  = s->p.gamma * pow(hypot(re, im), 3);
                double tr  = (g3 * re) * w + (gm * re) * s->p.w_15;
                double ti  = (g3 * im) * w + (gm * im) * s->p.w_15;
                o[2 * q]     = o[2 * q] - s->p.imag_time_dt * tr;
                o[2 * q + 1] = o[2 * q + 1] - s->p.imag_time_dt * ti;
            }
    memcpy(s->cpsi, s->cpsii, sizeof(double) * 2 * (size_t)nx * ny * nz);
}

/* CpuGrossPitaevskiSolver::real_fft_potential_half_step: cpu_solver.cpp:99-131. */
void gpeo_real_fft_potential_half_step(gpeo_solver *s) {
    const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
    const double w = s->p.n_atoms, dt_factor = s->p.real_time_dt / 2.;
    double *c = s->cpsi;
    for (int i = 1; i < nx - 1; i++)
        for (int j = 1; j < ny - 1; j++)
            for (int k = 1; k < nz - 1; k++) {
                size_t q       = IDX(s, i, j, k);
                double v_ext   = s->pote[q];
                double re      = c[2 * q], im = c[2 * q + 1];
                double density = re * re + im * im;
                double v_int   = (s->p.ggp11 - s->p.cdd / 3) * density * w +
                               s->p.gamma * pow(hypot(re, im), 3) * s->p.w_15;
                double total = v_ext + s->p.cdd * s->fi3d[q] + v_int;
                double sn, cs;
                sincos(-dt_factor * total, &sn, &cs);
                c[2 * q + 1] = re * sn + im * cs;
                c[2 * q]     = re * cs - im * sn;
            }
}

/* FFTWRealTimeSplitSolver::execute: fftw_split_solver.cpp:44-86. */
void gpeo_real_fft_kinetic_step(gpeo_solver *s) {
    const size_t N = (size_t)s->p.nx * s->p.ny * s->p.nz;
    memcpy(s->sp_r, s->cpsi, sizeof(double) * 2 * N);
    fftw_execute(s->sp_fwd);
    for (size_t t = 0; t < N; t++) {
        double sn, cs;
        sincos(s->kin[t], &sn, &cs);
        double ar = s->sp_k[2 * t], ai = s->sp_k[2 * t + 1];
        s->sp_k[2 * t]     = ar * cs - ai * sn;
        s->sp_k[2 * t + 1] = ar * sn + ai * cs;
    }
    fftw_execute(s->sp_bwd);
    const double norm_factor = 1.0 / (double)N;
    for (size_t t = 0; t < N; t++) {
        s->cpsi[2 * t]     = s->sp_r[2 * t] * norm_factor;
        s->cpsi[2 * t + 1] = s->sp_r[2 * t + 1] * norm_factor;
    }
}

/* CpuGrossPitaevskiSolver::calc_energy: cpu_solver.cpp:137-194.
 * out6 = {e_kin, e_pot, e_int, e_ext (dipolar), e_bmf, e_total}. */
void gpeo_calc_energy(gpeo_solver *s, double *out) {
    const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
    const double *c = s->cpsi;
    double e_kin = 0., e_pot = 0., e_int = 0., e_ext = 0., e_bmf = 0.;
    const double dx2 = pow(s->p.dx, 2), dy2 = pow(s->p.dy, 2), dz2 = pow(s->p.dz, 2);
    for (int i = 1; i < nx - 1; i++)
        for (int j = 1; j < ny - 1; j++)
            for (int k = 1; k < nz - 1; k++) {
                size_t q  = IDX(s, i, j, k);
                size_t xm = IDX(s, i - 1, j, k), xp = IDX(s, i + 1, j, k);
                size_t ym = IDX(s, i, j - 1, k), yp = IDX(s, i, j + 1, k);
                size_t zm = IDX(s, i, j, k - 1), zp = IDX(s, i, j, k + 1);
                double re = c[2 * q], im = c[2 * q + 1];
                double gxr = -((c[2 * xp] + c[2 * xm]) - 2. * re) / dx2;
                double gxi = -((c[2 * xp + 1] + c[2 * xm + 1]) - 2. * im) / dx2;
                double gyr = -((c[2 * yp] + c[2 * ym]) - 2. * re) / dy2;
                double gyi = -((c[2 * yp + 1] + c[2 * ym + 1]) - 2. * im) / dy2;
                double gzr = -((c[2 * zp] + c[2 * zm]) - 2. * re) / dz2;
                double gzi = -((c[2 * zp + 1] + c[2 * zm + 1]) - 2. * im) / dz2;
                double sr  = (gxr + gyr) + gzr;
                double si  = (gxi + gyi) + gzi;
                e_kin += sr * re - si * (-im);
                double nrm = re * re + im * im;
                e_pot += s->pote[q] * nrm;
                e_int += 0.5 * s->p.ggp11 * nrm * nrm;
                e_ext += 0.5 * s->p.cdd * s->fi3d[q] * nrm * s->p.n_atoms;
                e_ext -= s->p.cdd / 3. * pow(nrm, 2) / 2. * pow(s->p.n_atoms, 2);
                e_bmf += 2. / 5. * s->p.gamma * pow(hypot(re, im), 5);
            }
    e_kin *= s->p.dxdydz / (2 * s->p.m) * s->p.n_atoms;
    e_pot *= s->p.dxdydz * s->p.n_atoms;
    e_int *= s->p.dxdydz * pow(s->p.n_atoms, 2);
    e_ext *= s->p.dxdydz;
    e_bmf *= s->p.dxdydz * pow(s->p.n_atoms, 2.5);
    out[0] = e_kin;
    out[1] = e_pot;
    out[2] = e_int;
    out[3] = e_ext;
    out[4] = e_bmf;
    out[5] = e_kin + e_pot + e_int + e_ext + e_bmf;
}

/* AbstractGrossPitaevskiSolver::imag_time_iter: solver.cpp:99-105. */
void gpeo_imag_time_iter(gpeo_solver *s) {
    gpeo_calc_fi3d(s);
    gpeo_imag_iter_linear_step(s);
    gpeo_imag_iter_nonlinear_step(s);
    gpeo_calc_norm(s);
    gpeo_normalize(s);
}

/* AbstractGrossPitaevskiSolver::real_time_iter: solver.cpp:107-112. */
void gpeo_real_time_iter(gpeo_solver *s) {
    gpeo_real_fft_potential_half_step(s);
    gpeo_calc_fi3d(s);
    gpeo_real_fft_kinetic_step(s);
    gpeo_real_fft_potential_half_step(s);
}

void gpeo_imag_steps(gpeo_solver *s, long k) {
    for (long t = 0; t < k; ++t)
        gpeo_imag_time_iter(s);
}

/* calc_evolution's loop body without I/O: solver.cpp:75-78. */
void gpeo_real_steps(gpeo_solver *s, long k, long first_iter) {
    for (long t = 0; t < k; ++t) {
        if (!s->p.const_edd)
            gpeo_update_edd(&s->p, (unsigned)(first_iter + t));
        gpeo_real_time_iter(s);
    }
}
