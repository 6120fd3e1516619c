// Adapter harness -- TEST INFRASTRUCTURE ONLY.
//
// Links the reference's own, unmodified base class and driver code
// (AbstractGrossPitaevskiSolver in src/solver/solver.cpp, PhysicalParameters,
// SimulationContext, DataInitializer) with gpesolver_b200/adapter's
// B200GrossPitaevskiSolver and libgpe_b200.so into oracle/_ref/libgpe_adapter.so.
// The GPU tests then run the reference's own control flow -- imag_time_iter,
// real_time_iter and solve() (src/solver/solver.cpp:25-112) -- on the B200
// backend and compare against oracle/_ref/libgpe_ref.so (the same code on the
// reference's CPU backend).  This is the drop-in check: the reference's code
// calls the adapter's virtuals exactly as it calls its own backends'.
#include "b200_gpe_solver.hpp"
#include "initializer/initializer.hpp"
#include "manager/sim_mediator.hpp"
#include "ref_config.hpp"

#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

class AdapterSolver;

// Stands in for SimulationManager (src/manager/sim_manager.cpp): forwards the
// initializer's callbacks to the solver and keeps what the reference would
// write to files (checkpoints, energies) in memory.
class RecordingMediator : public AbstractSimulationMediator {
public:
    AdapterSolver *solver        = nullptr;
    DataInitializer *initializer = nullptr;
    std::vector<BECEnergies> energies;
    long checkpoints = 0;
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
};

class AdapterSolver : public B200GrossPitaevskiSolver {
public:
    AdapterSolver(AbstractSimulationMediator *m, int precision)
        : B200GrossPitaevskiSolver(m, precision) {}
    using AbstractGrossPitaevskiSolver::imag_time_iter;
    using AbstractGrossPitaevskiSolver::real_time_iter;
    using B200GrossPitaevskiSolver::calc_energy;
    using B200GrossPitaevskiSolver::export_data;
    CPUSolverData &buf() { return *buf_data; }
    const energies_t &energies() const { return ene; }
};

void RecordingMediator::on_data_loaded(const wavefunction_t &w) { solver->load_buffer(w); }
void RecordingMediator::on_data_initialized(const wavefunction_t &w) { solver->load_buffer(w); }
void RecordingMediator::on_pote_initialized(const potential_t &p) { solver->load_pote(p); }
void RecordingMediator::on_pote_changed(const potential_t &p) { solver->load_pote(p); }

struct State {
    RecordingMediator mediator;
    std::unique_ptr<AdapterSolver> solver;
    std::unique_ptr<DataInitializer> initializer;
};

std::unique_ptr<State> g_state;
std::string g_err;

template <class F> int guarded(F &&f) {
    if (!g_state)
        return (g_err = "no adapter state", 1);
    try {
        f();
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return 1;
    }
}

} // namespace

extern "C" {

const char *gpeadp_last_error(void) { return g_err.c_str(); }

// precision: 0 complex64, 1 complex128 (GPE_PREC_*).
int gpeadp_create(const gperef_config *c, int precision) {
    try {
        g_state.reset();
        gperef_apply_config(c);
        auto st                  = std::make_unique<State>();
        st->solver               = std::make_unique<AdapterSolver>(&st->mediator, precision);
        st->initializer          = std::make_unique<DataInitializer>(&st->mediator);
        st->mediator.solver      = st->solver.get();
        st->mediator.initializer = st->initializer.get();
        // SimulationManager::on_params_loaded (src/manager/sim_manager.cpp:50-58).
        st->solver->initialize();
        st->initializer->initialize_wavefunction();
        st->initializer->initialize_potential();
        g_state = std::move(st);
        return 0;
    } catch (const std::exception &e) {
        g_state.reset();
        g_err = e.what();
        return 1;
    }
}

void gpeadp_destroy(void) { g_state.reset(); }

// The base class's iteration functions (src/solver/solver.cpp:99-112); the RT
// ramp is applied first, as calc_evolution does (solver.cpp:76-77).
int gpeadp_imag_steps(long k) {
    return guarded([&] {
        for (long s = 0; s < k; ++s)
            g_state->solver->imag_time_iter();
    });
}

int gpeadp_real_steps(long k, long first_iter) {
    return guarded([&] {
        PhysicalParameters *p = PhysicalParameters::getInstance();
        for (long s = 0; s < k; ++s) {
            if (!p->const_edd)
                p->update_edd((unsigned)(first_iter + s));
            g_state->solver->real_time_iter();
        }
    });
}

// AbstractGrossPitaevskiSolver::solve (solver.cpp:25-46) with the given
// strategy: 0 IT, 1 RT, 2 FULL.
int gpeadp_solve(int strategy) {
    return guarded([&] {
        PhysicalParameters *p = PhysicalParameters::getInstance();
        p->calc_strategy.type = strategy == 0   ? CalcStrategy::Type::IMAGINARY_TIME
                                : strategy == 1 ? CalcStrategy::Type::REAL_TIME
                                                : CalcStrategy::Type::FULL;
        g_state->solver->solve();
    });
}

int gpeadp_export_psi(double *out) {
    return guarded([&] {
        g_state->solver->export_data();
        const wavefunction_t &w = g_state->solver->buf().cpsi;
        std::memcpy(out, w.get_data(), sizeof(double) * 2 * w.size());
    });
}

// {e_kin, e_pot, e_int, e_ext, e_bmf, e_total} from the adapter's calc_energy.
int gpeadp_energy(double *out) {
    return guarded([&] {
        g_state->solver->calc_energy();
        const energies_t &e = g_state->solver->energies();
        const double v[6]   = {e.e_kin, e.e_pot, e.e_int, e.e_ext, e.e_bmf, e.e_total};
        std::memcpy(out, v, sizeof(v));
    });
}

// What solve() handed to save_checkpoint / save_energies.
long gpeadp_checkpoints(void) { return g_state ? g_state->mediator.checkpoints : -1; }

long gpeadp_saved_energies(double *out, long max_rows) {
    if (!g_state)
        return -1;
    const auto &v = g_state->mediator.energies;
    const long n  = (long)v.size();
    for (long r = 0; r < n && r < max_rows; ++r) {
        const double row[6] = {v[r].e_kin, v[r].e_pot, v[r].e_int, v[r].e_ext, v[r].e_bmf, v[r].e_total};
        std::memcpy(out + 6 * r, row, sizeof(row));
    }
    return n;
}

} // extern "C"
