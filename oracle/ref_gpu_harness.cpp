// Reference GPU harness -- MEASUREMENT INFRASTRUCTURE ONLY.
//
// Compiled with the reference's own, unmodified GPU backend (GpuGrossPitaevskiSolver,
// its CUDA kernels and the cuFFT FP64 solvers: src/solver/cuda_solver/*,
// src/solver/fft_solvers/gpu/*) into oracle/_ref/libgpe_refgpu.so by
// oracle/Makefile (target refgpu), so that the reference's own GPU path can be
// timed on the same B200 beside this project's kernels.  It drives the solver
// through the reference's base-class iterations (imag_time_iter /
// real_time_iter, src/solver/solver.cpp:99-112) exactly as ref_harness.cpp
// drives the CPU backend.
#include "initializer/initializer.hpp"
#include "manager/sim_mediator.hpp"
#include "ref_config.hpp"
#include "solver/cuda_solver/gpu_solver.hpp"

#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <string>

namespace {

class GpuHarness;

class Mediator : public AbstractSimulationMediator {
public:
    GpuHarness *solver           = nullptr;
    DataInitializer *initializer = nullptr;
    void on_data_loaded(const wavefunction_t &) override;
    void on_data_initialized(const wavefunction_t &) override;
    void on_pote_initialized(const potential_t &) override;
    void on_pote_changed(const potential_t &) override;
    void on_params_loaded() override {}
    void request_load_from_binary(wavefunction_t &) override {}
    void request_load_from_text(wavefunction_t &) override {}
    void request_free_potential() override { initializer->change_potential("MEXICAN_FREE"); }
    void save_data(const wavefunction_t &) override {}
    void save_checkpoint(const wavefunction_t &) override {}
    void save_initial_state(const wavefunction_t &) override {}
    void save_energies(const energies_container_t &) override {}
};

class GpuHarness : public GpuGrossPitaevskiSolver {
public:
    explicit GpuHarness(AbstractSimulationMediator *m) : GpuGrossPitaevskiSolver(m) {}
    using AbstractGrossPitaevskiSolver::imag_time_iter;
    using AbstractGrossPitaevskiSolver::real_time_iter;
    using AbstractGrossPitaevskiSolver::calc_energy;
    using AbstractGrossPitaevskiSolver::export_data;
    CPUSolverData &buf() { return *buf_data; }
    const energies_t &energies() const { return ene; }
};

void Mediator::on_data_loaded(const wavefunction_t &w) { solver->load_buffer(w); }
void Mediator::on_data_initialized(const wavefunction_t &w) { solver->load_buffer(w); }
void Mediator::on_pote_initialized(const potential_t &p) { solver->load_pote(p); }
void Mediator::on_pote_changed(const potential_t &p) { solver->load_pote(p); }

struct State {
    Mediator mediator;
    std::unique_ptr<GpuHarness> solver;
    std::unique_ptr<DataInitializer> initializer;
};

std::unique_ptr<State> g_state;
std::string g_err;

} // namespace

extern "C" {

const char *gperefgpu_last_error(void) { return g_err.c_str(); }

int gperefgpu_create(const gperef_config *c) {
    try {
        g_state.reset();
        gperef_apply_config(c);
        auto st                  = std::make_unique<State>();
        st->solver               = std::make_unique<GpuHarness>(&st->mediator);
        st->initializer          = std::make_unique<DataInitializer>(&st->mediator);
        st->mediator.solver      = st->solver.get();
        st->mediator.initializer = st->initializer.get();
        st->solver->initialize();
        st->initializer->initialize_wavefunction();
        st->initializer->initialize_potential();
        g_state = std::move(st);
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return 1;
    }
}

void gperefgpu_destroy(void) { g_state.reset(); }

int gperefgpu_change_potential(const char *key) {
    if (!g_state) return 1;
    g_state->initializer->change_potential(std::string(key));
    return 0;
}

int gperefgpu_imag_steps(long k) {
    if (!g_state) return 1;
    for (long s = 0; s < k; ++s)
        g_state->solver->imag_time_iter();
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

int gperefgpu_real_steps(long k, long first_iter) {
    if (!g_state) return 1;
    PhysicalParameters *p = PhysicalParameters::getInstance();
    for (long s = 0; s < k; ++s) {
        if (!p->const_edd)
            p->update_edd((unsigned)(first_iter + s));
        g_state->solver->real_time_iter();
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

int gperefgpu_export_psi(double *out) {
    if (!g_state) return 1;
    g_state->solver->export_data();
    const wavefunction_t &w = g_state->solver->buf().cpsi;
    std::memcpy(out, w.get_data(), sizeof(double) * 2 * w.size());
    return 0;
}

int gperefgpu_energy(double *out) {
    if (!g_state) return 1;
    g_state->solver->calc_energy();
    const energies_t &e = g_state->solver->energies();
    const double v[6]   = {e.e_kin, e.e_pot, e.e_int, e.e_ext, e.e_bmf, e.e_total};
    std::memcpy(out, v, sizeof(v));
    return 0;
}

} // extern "C"
