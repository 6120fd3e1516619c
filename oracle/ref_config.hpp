// Parameter set-up shared by the reference harnesses -- TEST INFRASTRUCTURE ONLY.
//
// gperef_config mirrors the gpe_params.json fields the reference loads;
// gperef_apply_config fills the reference's PhysicalParameters singleton from it
// and runs what SimulationManager::on_params_loaded runs before the solver is
// created (src/manager/sim_manager.cpp:50-58).
#pragma once

#include "context/context.hpp"
#include "parameters/parameters.hpp"
#include "units.hpp"

#include <string>

extern "C" {
// Mirror of the gpe_params.json fields the reference loads
// (src/filemanager/file_manager.cpp:436-541), in the file's units (nm, Da, Hz).
struct gperef_config {
    int nx, ny, nz;
    double dx_nm, dy_nm, dz_nm;
    double m_da;
    double n_atoms;
    double omega_x_hz, omega_y_hz, omega_z_hz;
    double dd_nm;
    int const_edd;
    double edd, edd_start, edd_stop;
    long iter_imag, iter_real;
    int init_strategy; // 0 COS, 1 GAUSS, 2 MULTIPLE_GAUSS, 3 SETUP_GAUSS, 4 none (load later)
    int n_gauss_max;
    int bec_droplets_x, bec_droplets_y, bec_droplets_z;
    int fftw_n_threads;
    char pote_key[32];
};
}

inline void gperef_apply_config(const gperef_config *c) {
    PhysicalParameters *p = PhysicalParameters::getInstance();
    // Same conversions as FileManager::load_box / load_simulation / load_potential.
    p->dx = UnitConverter::len_nm_to_au(c->dx_nm);
    p->dy = UnitConverter::len_nm_to_au(c->dy_nm);
    p->dz = UnitConverter::len_nm_to_au(c->dz_nm);
    p->nx = c->nx;
    p->ny = c->ny;
    p->nz = c->nz;
    p->iter_imag = (size_t)c->iter_imag;
    p->iter_real = (size_t)c->iter_real;
    p->n_atoms   = c->n_atoms;
    p->m         = UnitConverter::mass_Da_to_au(c->m_da);
    p->const_edd = c->const_edd != 0;
    if (p->const_edd) {
        p->edd = c->edd;
    } else {
        p->edd_start = c->edd_start;
        p->edd_stop  = c->edd_stop;
        // The reference leaves edd uninitialised when only a ramp is given
        // (src/parameters/parameters.hpp:120); the harness defines it as edd_start.
        p->edd = c->edd_start;
    }
    p->fftw_n_threads = c->fftw_n_threads > 0 ? c->fftw_n_threads : 4;
    p->pote_key       = std::string(c->pote_key);
    p->dd             = UnitConverter::len_nm_to_au(c->dd_nm);
    p->omega_x        = UnitConverter::freq_Hz_to_au(c->omega_x_hz);
    p->omega_y        = UnitConverter::freq_Hz_to_au(c->omega_y_hz);
    p->omega_z        = UnitConverter::freq_Hz_to_au(c->omega_z_hz);
    p->n_gauss_max    = c->n_gauss_max;
    p->bec_droplets_x = c->bec_droplets_x;
    p->bec_droplets_y = c->bec_droplets_y;
    p->bec_droplets_z = c->bec_droplets_z;
    switch (c->init_strategy) {
    case 0: p->init_strategy.type = InitializationOption::Type::COS; break;
    case 1: p->init_strategy.type = InitializationOption::Type::GAUSS; break;
    case 2: p->init_strategy.type = InitializationOption::Type::MULTIPLE_GAUSS; break;
    case 3: p->init_strategy.type = InitializationOption::Type::SETUP_GAUSS; break;
    default: break;
    }

    // SimulationManager::on_params_loaded (src/manager/sim_manager.cpp:50-58).
    p->init_parameters();
    SimulationContext::getInstance()->initialize();
}
