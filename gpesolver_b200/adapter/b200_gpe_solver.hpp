// B200GrossPitaevskiSolver -- the gpe_b200 backend behind GPESolver's
// AbstractGrossPitaevskiSolver (src/solver/solver.hpp:17-72).
//
// This file and b200_gpe_solver.cpp are meant to be added to GPESolver's own
// source tree (src/solver/b200_solver/) and selected by SolverFactory
// (src/solver/solver_factory.hpp:12-21) in place of GpuGrossPitaevskiSolver
// (src/solver/cuda_solver/gpu_solver.hpp:7-31).  They include only the
// reference's headers and include/gpe_b200.h, and link against libgpe_b200.so.
//
// Every pure virtual maps onto one gpe_* call.  The device holds psi, phi and V
// for the whole run; buf_data (the base class's CPU copy) is touched only by
// import_data / import_pote / export_data, as with the reference's GPU backend.
//
// With GPE_B200_FUSED_LOOPS defined, calc_initial_state / calc_evolution are
// overridden as well and run the iterations between two checkpoints as one
// fused device call (gpe_imag_steps / gpe_real_steps).  That needs those two
// methods declared virtual in solver.hpp:42-43; without the macro the adapter
// compiles against the unmodified header and the base class's loops drive the
// virtuals one by one.
#ifndef B200_GPE_SOLVER_HPP
#define B200_GPE_SOLVER_HPP

#include "gpe_b200.h"
#include "solver/solver.hpp"

class B200GrossPitaevskiSolver : public AbstractGrossPitaevskiSolver {
public:
    //! precision: GPE_PREC_C64 (complex64 fields, the fast path) or GPE_PREC_C128.
    //! device: CUDA ordinal the handle lives on.
    explicit B200GrossPitaevskiSolver(AbstractSimulationMediator *mediator,
                                      int precision = GPE_PREC_C64, int device = 0);
    // AbstractGrossPitaevskiSolver has no virtual destructor: delete through the
    // derived type, or add `virtual ~AbstractGrossPitaevskiSolver() = default;`
    // to solver.hpp so that SolverFactory's unique_ptr releases the handle.
    ~B200GrossPitaevskiSolver();

    B200GrossPitaevskiSolver(const B200GrossPitaevskiSolver &)            = delete;
    B200GrossPitaevskiSolver &operator=(const B200GrossPitaevskiSolver &) = delete;

    //! The underlying handle (null before initialize()).
    gpe_handle *handle() const { return m_handle; }

protected:
    void calc_energy() override;
    void init_containers() override;
    void calc_fi3d() override;
    void calc_norm() override;
    void normalize() override;
    void imag_iter_linear_step() override;
    void imag_iter_nonlinear_step() override;
    void real_fft_potential_half_step() override;
    void real_fft_kinetic_step() override;
    void prepare_fft() override;
    void export_data() override;
    void import_data() override;
    void import_pote() override;

#ifdef GPE_B200_FUSED_LOOPS
    void calc_initial_state() override;
    void calc_evolution() override;
#endif

private:
    gpe_handle *m_handle = nullptr;
    int m_precision;
    int m_device;
    bool m_loaded = false; // a wavefunction has been imported
    double m_ggp11 = 0, m_gamma = 0; // coefficients the handle holds

    void check(int rc, const char *what) const;
    void sync_coeffs();
    gpe_params make_params() const;
};

#endif
