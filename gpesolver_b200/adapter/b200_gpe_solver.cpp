// B200GrossPitaevskiSolver: AbstractGrossPitaevskiSolver's virtuals on the gpe_b200
// C ABI.  Each method names the reference method it replaces
// (src/solver/cuda_solver/gpu_solver.cpp, src/solver/cpu_solver/cpu_solver.cpp).
#include "b200_gpe_solver.hpp"

#include "output.hpp"
#include "units.hpp"

#include <algorithm>
#include <stdexcept>
#include <string>

namespace {

size_t grid_points(const PhysicalParameters *p) {
    return (size_t)p->nx * (size_t)p->ny * (size_t)p->nz;
}

} // namespace

B200GrossPitaevskiSolver::B200GrossPitaevskiSolver(AbstractSimulationMediator *mediator,
                                                   int precision, int device)
    : AbstractGrossPitaevskiSolver(mediator), m_precision(precision), m_device(device) {}

B200GrossPitaevskiSolver::~B200GrossPitaevskiSolver() {
    if (m_handle)
        gpe_destroy(m_handle);
}

void B200GrossPitaevskiSolver::check(int rc, const char *what) const {
    if (rc != GPE_OK)
        throw std::runtime_error(std::string("gpe_b200 ") + what + ": " + gpe_last_error());
}

// The PhysicalParameters fields the backend reads, as init_parameters / update_edd
// left them (src/parameters/parameters.cpp:37-59).
gpe_params B200GrossPitaevskiSolver::make_params() const {
    gpe_params p{};
    p.nx           = params->nx;
    p.ny           = params->ny;
    p.nz           = params->nz;
    p.dx           = params->dx;
    p.dy           = params->dy;
    p.dz           = params->dz;
    p.m            = params->m;
    p.n_atoms      = params->n_atoms;
    p.add          = params->add;
    p.cdd          = params->cdd;
    p.ggp11        = params->ggp11;
    p.gamma        = params->gamma;
    p.w_15         = params->w_15;
    p.real_time_dt = params->real_time_dt;
    p.imag_time_dt = params->imag_time_dt;
    p.const_edd    = params->const_edd ? 1 : 0;
    p.edd          = params->edd;
    p.edd_start    = params->const_edd ? params->edd : params->edd_start;
    p.edd_stop     = params->const_edd ? params->edd : params->edd_stop;
    p.iter_real    = (long)params->iter_real;
    p.precision    = m_precision;
    p.device       = m_device;
    p.schedule     = GPE_SCHED_AUTO;
    return p;
}

// update_edd changes ggp11 and gamma on the host between iterations
// (src/solver/solver.cpp:76-77); the handle takes them before the next use.
void B200GrossPitaevskiSolver::sync_coeffs() {
    if (params->ggp11 != m_ggp11 || params->gamma != m_gamma) {
        check(gpe_set_coeffs(m_handle, params->ggp11, params->gamma), "set_coeffs");
        m_ggp11 = params->ggp11;
        m_gamma = params->gamma;
    }
}

// GpuGrossPitaevskiSolver::init_containers (gpu_solver.cpp:26-32): device fields,
// FFT plans and the V_dd / kinetic tables, all inside gpe_create.
void B200GrossPitaevskiSolver::init_containers() {
    if (m_handle) {
        gpe_destroy(m_handle);
        m_handle = nullptr;
    }
    const gpe_params p = make_params();
    check(gpe_create(&p, &m_handle), "create");
    m_ggp11  = params->ggp11;
    m_gamma  = params->gamma;
    m_loaded = false;
}

// prepare_fft (gpu_solver.cpp:34-38): planned by gpe_create.
void B200GrossPitaevskiSolver::prepare_fft() {}

// import_data (gpu_solver.cpp:141-148): psi and psii take buf_data's values.
void B200GrossPitaevskiSolver::import_data() {
    const size_t n = grid_points(params);
    check(gpe_import_psi(m_handle, reinterpret_cast<const double *>(buf_data->cpsi.get_data()), n),
          "import_psi");
    m_loaded = true;
}

// import_pote (gpu_solver.cpp:150-152).
void B200GrossPitaevskiSolver::import_pote() {
    check(gpe_load_potential(m_handle, buf_data->pote.get_data(), grid_points(params)),
          "load_potential");
}

// export_data (gpu_solver.cpp:136-139): psi into buf_data->cpsi.
void B200GrossPitaevskiSolver::export_data() {
    check(gpe_export_psi(m_handle, reinterpret_cast<double *>(buf_data->cpsi.get_data()),
                         grid_points(params)),
          "export_psi");
}

void B200GrossPitaevskiSolver::calc_fi3d() { check(gpe_calc_fi3d(m_handle), "calc_fi3d"); }

void B200GrossPitaevskiSolver::imag_iter_linear_step() {
    sync_coeffs();
    check(gpe_imag_iter_linear_step(m_handle), "imag_iter_linear_step");
}

void B200GrossPitaevskiSolver::imag_iter_nonlinear_step() {
    check(gpe_imag_iter_nonlinear_step(m_handle), "imag_iter_nonlinear_step");
}

// initialize() (solver.cpp:15-23) normalises before any wavefunction is loaded;
// the reference divides zeros by zero there and load_buffer overwrites the
// result.  The adapter skips both calls until import_data has run.
void B200GrossPitaevskiSolver::calc_norm() {
    if (!m_loaded)
        return;
    check(gpe_calc_norm(m_handle, &xnorma), "calc_norm");
}

void B200GrossPitaevskiSolver::normalize() {
    if (!m_loaded)
        return;
    check(gpe_normalize(m_handle), "normalize");
}

void B200GrossPitaevskiSolver::real_fft_potential_half_step() {
    sync_coeffs();
    check(gpe_real_fft_potential_half_step(m_handle), "real_fft_potential_half_step");
}

void B200GrossPitaevskiSolver::real_fft_kinetic_step() {
    check(gpe_real_fft_kinetic_step(m_handle), "real_fft_kinetic_step");
}

// calc_energy (cpu_solver.cpp:137-194): the same six terms, appended to enes.
void B200GrossPitaevskiSolver::calc_energy() {
    sync_coeffs();
    double e[6];
    check(gpe_calc_energy(m_handle, e), "calc_energy");
    ene.e_kin   = e[0];
    ene.e_pot   = e[1];
    ene.e_int   = e[2];
    ene.e_ext   = e[3];
    ene.e_bmf   = e[4];
    ene.e_total = e[5];
    enes.emplace_back(ene);
}

#ifdef GPE_B200_FUSED_LOOPS
// calc_initial_state (solver.cpp:48-70) with the iterations between two
// checkpoints (every 100th) run as one fused device call.
void B200GrossPitaevskiSolver::calc_initial_state() {
    OutputFormatter::printInfo("Starting imaginary time evolution");
    const size_t last = params->iter_imag;
    for (size_t iter = 0; iter <= last;) {
        const size_t ckpt = (iter + 99) / 100 * 100; // first checkpoint at or after iter
        const size_t stop = std::min(ckpt, last);
        sync_coeffs();
        check(gpe_imag_steps(m_handle, (long)(stop - iter + 1)), "imag_steps");
        if (stop == ckpt) {
            export_data();
            p_mediator->save_checkpoint(buf_data->cpsi);
            summarize_imag_iter();
            calc_energy();
        }
        iter = stop + 1;
    }
    OutputFormatter::printInfo("Imaginary time evolution completed");
    OutputFormatter::printBorderLine();
    OutputFormatter::printBoxedMessage("Minimized energy [meV]: ",
                                       UnitConverter::ene_au_to_meV(ene.e_total));
    OutputFormatter::printBorderLine();
    p_mediator->save_energies(enes);
}

// calc_evolution (solver.cpp:72-97): every 1000th iteration is a checkpoint; the
// edd ramp (update_edd before each iteration) runs inside gpe_real_steps.
void B200GrossPitaevskiSolver::calc_evolution() {
    OutputFormatter::printInfo("Starting real time evolution");
    const size_t last = params->iter_real;
    for (size_t iter = 0; iter <= last;) {
        const size_t ckpt = (iter + 999) / 1000 * 1000;
        const size_t stop = std::min(ckpt, last);
        sync_coeffs();
        check(gpe_real_steps(m_handle, (long)(stop - iter + 1), (long)iter), "real_steps");
        if (!params->const_edd) {
            params->update_edd((unsigned)stop); // the host copy follows the device
            m_ggp11 = params->ggp11;
            m_gamma = params->gamma;
        }
        if (stop == ckpt) {
            export_data();
            p_mediator->save_checkpoint(buf_data->cpsi);
            summarize_real_iter();
            calc_energy();
        }
        iter = stop + 1;
    }
    OutputFormatter::printInfo("Real time evolution completed");
    OutputFormatter::printBorderLine();
    OutputFormatter::printBoxedMessage("Finished on energy [meV]: ",
                                       UnitConverter::ene_au_to_meV(ene.e_total));
    OutputFormatter::printBorderLine();
    p_mediator->save_data(buf_data->cpsi);
    p_mediator->save_energies(enes);
}
#endif
