// Reference harness -- TEST INFRASTRUCTURE ONLY (part of the oracle).
//
// Compiled together with the reference's own, unmodified CPU sources (see
// oracle/Makefile) into oracle/_ref/libgpe_ref.so.  It drives the reference's
// CpuGrossPitaevskiSolver exactly as its SimulationManager does
// (src/manager/sim_manager.cpp:50-80), but without file output, and exposes a
// small C ABI so that Python tests and the bench's CPU baseline can step it one
// iteration at a time and read back psi, phi (fi3d), V and the energies.
//
// Nothing here changes the reference's arithmetic: every number comes from the
// reference's own functions (imag_time_iter / real_time_iter at
// src/solver/solver.cpp:99-112, calc_energy at
// src/solver/cpu_solver/cpu_solver.cpp:137-194, DataInitializer at
// src/initializer/initializer.cpp, PotentialRegistry at
// src/parameters/potentials.hpp:76-157), linked against the FP64 FFTW-API shim in
// oracle/fftw_shim.
#include "context/context.hpp"
#include "filemanager/file_manager.hpp"
#include "initializer/initializer.hpp"
#include "manager/sim_mediator.hpp"
#include "parameters/parameters.hpp"
#include "solver/cpu_solver/cpu_solver.hpp"
#include "solver/fft_solvers/cpu/fftw_abstract_cpu_solver.hpp"
#include "ref_config.hpp"
#include "units.hpp"

#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

class HarnessSolver;

class NullMediator : public AbstractSimulationMediator {
public:
    HarnessSolver *solver          = nullptr;
    DataInitializer *initializer   = nullptr;
    void on_data_loaded(const wavefunction_t &) override;
    void on_data_initialized(const wavefunction_t &) override;
    void on_pote_initialized(const potential_t &) override;
    void on_pote_changed(const potential_t &) override;
    void on_params_loaded() override {}
    void request_load_from_binary(wavefunction_t &) override {}
    void request_load_from_text(wavefunction_t &) override {}
    void request_free_potential() override { initializer->change_potential("MEXICAN_FREE"); }
    void save_data(const wavefunction_t &) override {}
    void save_checkpoint(const wavefunction_t &) override { ++checkpoints; }
    void save_initial_state(const wavefunction_t &) override {}
    void save_energies(const energies_container_t &e) override { energies = e; }
    std::vector<BECEnergies> energies;
    long checkpoints = 0;
};

// Exposes the protected step functions of the reference's base class and the
// (privately overridden) virtuals of the CPU backend.  The using-declarations
// re-expose the base-class names; calls still dispatch virtually to
// CpuGrossPitaevskiSolver's implementations.
class HarnessSolver : public CpuGrossPitaevskiSolver {
public:
    explicit HarnessSolver(AbstractSimulationMediator *m) : CpuGrossPitaevskiSolver(m) {}
    using AbstractGrossPitaevskiSolver::calc_energy;
    using AbstractGrossPitaevskiSolver::calc_fi3d;
    using AbstractGrossPitaevskiSolver::calc_norm;
    using AbstractGrossPitaevskiSolver::export_data;
    using AbstractGrossPitaevskiSolver::imag_iter_linear_step;
    using AbstractGrossPitaevskiSolver::imag_iter_nonlinear_step;
    using AbstractGrossPitaevskiSolver::imag_time_iter;
    using AbstractGrossPitaevskiSolver::normalize;
    using AbstractGrossPitaevskiSolver::real_fft_kinetic_step;
    using AbstractGrossPitaevskiSolver::real_fft_potential_half_step;
    using AbstractGrossPitaevskiSolver::real_time_iter;

    CPUSolverData &buf() { return *buf_data; }
    FFTWAbstractCPUSolver *poisson() { return dynamic_cast<FFTWAbstractCPUSolver *>(poisson_solver.get()); }
    const energies_t &energies() const { return ene; }
    double norm() const { return xnorma; }
};

// Reads the protected field pointers of the reference's FFTW solvers (they point
// at the CPU backend's private working arrays, src/solver/cpu_solver/cpu_solver.cpp:196-199)
// through a pointer-to-member formed in a derived class.
struct FieldPeek : FFTWAbstractCPUSolver {
    static potential_t *fi3d_of(FFTWAbstractCPUSolver *s) { return s->*(&FieldPeek::fi3d); }
    static wavefunction_t *psi_of(FFTWAbstractCPUSolver *s) { return s->*(&FieldPeek::psi); }
};

void NullMediator::on_data_loaded(const wavefunction_t &w) { solver->load_buffer(w); }
void NullMediator::on_data_initialized(const wavefunction_t &w) { solver->load_buffer(w); }
void NullMediator::on_pote_initialized(const potential_t &p) { solver->load_pote(p); }
void NullMediator::on_pote_changed(const potential_t &p) { solver->load_pote(p); }

struct State {
    NullMediator mediator;
    std::unique_ptr<HarnessSolver> solver;
    std::unique_ptr<DataInitializer> initializer;
    // Copies the harness keeps of what the reference's containers hold, because
    // m_data (the CPU backend's working copy) is private; export_data() copies
    // cpsi into buf_data, and phi / V are tracked through the calls that set them.
};

std::unique_ptr<State> g_state;
std::string g_err;

int fail(const std::exception &e) {
    g_err = e.what();
    return 1;
}

} // namespace

extern "C" {

const char *gperef_last_error(void) { return g_err.c_str(); }

int gperef_create(const gperef_config *c) {
    try {
        g_state.reset();
        gperef_apply_config(c);
        auto st                 = std::make_unique<State>();
        st->solver              = std::make_unique<HarnessSolver>(&st->mediator);
        st->initializer         = std::make_unique<DataInitializer>(&st->mediator);
        st->mediator.solver      = st->solver.get();
        st->mediator.initializer = st->initializer.get();
        st->solver->initialize();
        if (c->init_strategy >= 0 && c->init_strategy <= 3)
            st->initializer->initialize_wavefunction();
        st->initializer->initialize_potential();
        g_state = std::move(st);
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

void gperef_destroy(void) { g_state.reset(); }

// Coefficients derived by PhysicalParameters::init_parameters / update_edd:
// out = {m, dx, dy, dz, cdd, ggp11, gamma, w_15, aa, b, dd, omega_x, omega_y, omega_z, edd}.
int gperef_coefficients(double *out) {
    PhysicalParameters *p = PhysicalParameters::getInstance();
    double v[15] = {p->m,    p->dx,  p->dy, p->dz, p->cdd,     p->ggp11,   p->gamma,  p->w_15,
                    p->aa,   p->b,   p->dd, p->omega_x, p->omega_y, p->omega_z, p->edd};
    std::memcpy(out, v, sizeof(v));
    return 0;
}

int gperef_update_edd(long iter) {
    PhysicalParameters::getInstance()->update_edd((unsigned)iter);
    return 0;
}

int gperef_load_psi(const double *psi_c128) {
    if (!g_state) return 1;
    PhysicalParameters *p = PhysicalParameters::getInstance();
    wavefunction_t w(p->nx, p->ny, p->nz);
    std::memcpy(w.get_data(), psi_c128, sizeof(double) * 2 * w.size());
    g_state->solver->load_buffer(w);
    return 0;
}

int gperef_load_pote(const double *v) {
    if (!g_state) return 1;
    PhysicalParameters *p = PhysicalParameters::getInstance();
    potential_t pot(p->nx, p->ny, p->nz);
    std::memcpy(pot.get_data(), v, sizeof(double) * pot.size());
    g_state->solver->load_pote(pot);
    return 0;
}

// Potential switch used by the FS strategy (src/solver/solver.cpp:114-116,
// src/manager/sim_manager.cpp:78-80, src/initializer/initializer.cpp:250-255).
int gperef_change_potential(const char *key) {
    if (!g_state) return 1;
    try {
        g_state->initializer->change_potential(std::string(key));
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// Full reference iterations: imag_time_iter / real_time_iter
// (src/solver/solver.cpp:99-112); RT applies the edd ramp first as
// calc_evolution does (src/solver/solver.cpp:76-77).
int gperef_imag_steps(long k) {
    if (!g_state) return 1;
    for (long s = 0; s < k; ++s)
        g_state->solver->imag_time_iter();
    return 0;
}

int gperef_real_steps(long k, long first_iter) {
    if (!g_state) return 1;
    PhysicalParameters *p = PhysicalParameters::getInstance();
    for (long s = 0; s < k; ++s) {
        if (!p->const_edd)
            p->update_edd((unsigned)(first_iter + s));
        g_state->solver->real_time_iter();
    }
    return 0;
}

// AbstractGrossPitaevskiSolver::solve (src/solver/solver.cpp:25-46) with the
// given strategy: 0 IT, 1 RT, 2 FULL.
int gperef_solve(int strategy) {
    if (!g_state) return 1;
    try {
        PhysicalParameters *p = PhysicalParameters::getInstance();
        p->calc_strategy.type = strategy == 0   ? CalcStrategy::Type::IMAGINARY_TIME
                                : strategy == 1 ? CalcStrategy::Type::REAL_TIME
                                                : CalcStrategy::Type::FULL;
        g_state->solver->solve();
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// What solve() handed to save_checkpoint / save_energies.
long gperef_checkpoints(void) { return g_state ? g_state->mediator.checkpoints : -1; }

long gperef_saved_energies(double *out, long max_rows) {
    if (!g_state) return -1;
    const auto &v = g_state->mediator.energies;
    const long n  = (long)v.size();
    for (long r = 0; r < n && r < max_rows; ++r) {
        const double row[6] = {v[r].e_kin, v[r].e_pot, v[r].e_int, v[r].e_ext, v[r].e_bmf, v[r].e_total};
        std::memcpy(out + 6 * r, row, sizeof(row));
    }
    return n;
}

// Individual virtuals, for per-operation parity checks.
int gperef_op(int which) {
    if (!g_state) return 1;
    HarnessSolver &s = *g_state->solver;
    switch (which) {
    case 0: s.calc_fi3d(); break;
    case 1: s.imag_iter_linear_step(); break;
    case 2: s.imag_iter_nonlinear_step(); break;
    case 3: s.calc_norm(); break;
    case 4: s.normalize(); break;
    case 5: s.real_fft_potential_half_step(); break;
    case 6: s.real_fft_kinetic_step(); break;
    case 7: s.calc_energy(); break;
    default: return 2;
    }
    return 0;
}

double gperef_norm(void) { return g_state ? g_state->solver->norm() : 0.0; }

// psi as interleaved (re, im) FP64, reference layout (i*ny + j)*nz + k.
int gperef_export_psi(double *out) {
    if (!g_state) return 1;
    g_state->solver->export_data();
    const wavefunction_t &w = g_state->solver->buf().cpsi;
    std::memcpy(out, w.get_data(), sizeof(double) * 2 * w.size());
    return 0;
}

// The dipolar field phi (m_data.fi3d) as last computed by calc_fi3d.
int gperef_export_fi3d(double *out) {
    if (!g_state) return 1;
    const potential_t *f = FieldPeek::fi3d_of(g_state->solver->poisson());
    std::memcpy(out, f->get_data(), sizeof(double) * f->size());
    return 0;
}

// The working psi (m_data.cpsi) without going through export_data.
int gperef_peek_psi(double *out) {
    if (!g_state) return 1;
    const wavefunction_t *w = FieldPeek::psi_of(g_state->solver->poisson());
    std::memcpy(out, w->get_data(), sizeof(double) * 2 * w->size());
    return 0;
}

// The potential last loaded into the solver (buf_data->pote).
int gperef_export_pote(double *out) {
    if (!g_state) return 1;
    const potential_t &v = g_state->solver->buf().pote;
    std::memcpy(out, v.get_data(), sizeof(double) * v.size());
    return 0;
}

// The reference's FileManager writers and reader (src/filemanager/file_manager.cpp:81-112,
// 251-290, 387-401, 404-434), on the harness's current psi / potential / energies.
// `name` has no extension (the writer appends it); energies go to
// energy.gpe.dat in the working directory.
int gperef_save_binary(const char *name) {
    if (!g_state) return 1;
    try {
        FileManager fm(&g_state->mediator);
        g_state->solver->export_data();
        fm.save_to_binary_file(g_state->solver->buf().cpsi, name);
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

int gperef_save_text(const char *name) {
    if (!g_state) return 1;
    try {
        FileManager fm(&g_state->mediator);
        g_state->solver->export_data();
        fm.save_to_text_file(g_state->solver->buf().cpsi, name);
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

int gperef_save_pote_text(const char *name) {
    if (!g_state) return 1;
    try {
        FileManager fm(&g_state->mediator);
        fm.save_pote_to_text_file(g_state->solver->buf().pote, name);
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

int gperef_save_energies(void) {
    if (!g_state) return 1;
    try {
        FileManager fm(&g_state->mediator);
        fm.save_energies(g_state->mediator.energies);
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// FileManager::load_from_binary_file (file_manager.cpp:292-335) into out (2n doubles).
int gperef_load_binary(const char *name, double *out) {
    if (!g_state) return 1;
    try {
        FileManager fm(&g_state->mediator);
        fm.load_from_binary_file(name, [&](wavefunction_t &w) {
            std::memcpy(out, w.get_data(), sizeof(double) * 2 * w.size());
        });
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// {e_kin, e_pot, e_int, e_ext (dipolar), e_bmf, e_total} after calc_energy.
int gperef_energy(double *out) {
    if (!g_state) return 1;
    g_state->solver->calc_energy();
    const energies_t &e = g_state->solver->energies();
    out[0] = e.e_kin;
    out[1] = e.e_pot;
    out[2] = e.e_int;
    out[3] = e.e_ext;
    out[4] = e.e_bmf;
    out[5] = e.e_total;
    return 0;
}

} // extern "C"
