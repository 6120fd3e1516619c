// Device-side initial state and trap potential (FP64), for callers that build
// many solves (parameter sweeps) and would otherwise spend their start-up in
// host loops and host-to-device copies.
//
// The arithmetic follows the reference's host functions operation by
// operation, with every product, sum and quotient rounded separately
// (__dmul_rn / __dadd_rn / __ddiv_rn: no fused multiply-add contraction), so
// that a potential comes out bit-identical to PotentialRegistry's
// (src/parameters/potentials.hpp:76-157).  The initial states use exp / cos,
// which neither the host library nor CUDA rounds correctly: those agree to an
// ulp or two.
#pragma once

#include <cuda_runtime.h>

namespace gpe {

struct InitGeom {
    int nx, ny, nz;
    double dx, dy, dz;
};

// Potential ids in the reference's registration order (potentials.hpp:76-157).
enum { POT_HARMONIC = 0, POT_MEXICAN, POT_MEXICAN_FREE, POT_CYLINDRICAL, POT_FREE, POT_MEXICAN_ASYMETRIC,
       POT_MEXICAN_ASYMETRIC_FREE, POT_COUNT };

struct PotCoef {
    int key;
    double m, wx, wy, wz, aa, b;
    double slope; // MEXICAN_ASYMETRIC*: (0.25 / conv) / dd, computed on the host
};

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dq(double a, double b) { return __ddiv_rn(a, b); }

// SimulationContext::initialize (src/context/context.cpp:17-34):
// coordinate i = (i - n/2) * d, the integer difference converted first.
__device__ __forceinline__ double coord(int i, int n, double d) { return dm((double)(i - n / 2), d); }

// 0.5 * m * pow(c, 2) * pow(w, 2), left to right
__device__ __forceinline__ double half_m_c2_w2(double m, double c, double w) {
    return dm(dm(dm(0.5, m), dm(c, c)), dm(w, w));
}

// DataInitializer::init_pote (src/initializer/initializer.cpp:229-248): the
// registry function takes int coordinates (initializer.hpp:37), so each
// coordinate is truncated toward zero before the potential sees it.
__global__ void k_init_potential(double *__restrict__ V, InitGeom g, PotCoef p) {
    const size_t N = (size_t)g.nx * g.ny * g.nz;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N; q += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(q % g.nz);
        const int j = (int)((q / g.nz) % g.ny);
        const int i = (int)(q / ((size_t)g.nz * g.ny));
        const double x = (double)(int)coord(i, g.nx, g.dx);
        const double y = (double)(int)coord(j, g.ny, g.dy);
        const double z = (double)(int)coord(k, g.nz, g.dz);
        const double vz = half_m_c2_w2(p.m, z, p.wz);
        double v;
        switch (p.key) {
        case POT_HARMONIC:
            v = da(da(half_m_c2_w2(p.m, x, p.wx), half_m_c2_w2(p.m, y, p.wy)), vz);
            break;
        case POT_MEXICAN:
        case POT_MEXICAN_ASYMETRIC: {
            const double x2 = dm(x, x);
            double vx       = da(dm(-p.b, x2), dm(p.aa, dm(x2, x2)));
            if (p.key == POT_MEXICAN_ASYMETRIC)
                vx = ds(vx, dm(p.slope, x));
            v = da(da(vx, half_m_c2_w2(p.m, y, p.wy)), vz);
            break;
        }
        case POT_MEXICAN_FREE:
        case POT_MEXICAN_ASYMETRIC_FREE: {
            const double x2 = dm(x, x);
            double vx       = dm(p.aa, dm(x2, x2));
            if (p.key == POT_MEXICAN_ASYMETRIC_FREE)
                vx = ds(vx, dm(p.slope, x));
            v = da(da(vx, half_m_c2_w2(p.m, y, p.wy)), vz);
            break;
        }
        case POT_CYLINDRICAL: {
            const double r = __dsqrt_rn(da(dm(x, x), dm(y, y)));
            v = da(half_m_c2_w2(p.m, r, dq(da(p.wy, p.wx), 2.)), vz);
            break;
        }
        default: // POT_FREE
            v = vz;
            break;
        }
        V[q] = v;
    }
}

// Initial-state strategies (src/parameters/complex_param.hpp:57-97).
enum { INIT_COS = 0, INIT_GAUSS, INIT_MULTIPLE_GAUSS, INIT_SETUP_GAUSS, INIT_COUNT };

constexpr int kMaxGaussCentres = 64;

struct PsiCoef {
    int strategy;
    double sx, sy, sz;  // Gaussian widths (GAUSS: L/10, multiple / setup: L/20)
    double rrr, dd;     // COS: int(nx/2) dx and the x shift
    int ncent;          // number of Gaussian centres
    int zcent;          // SETUP_GAUSS: centres carry a z coordinate
    double cx[kMaxGaussCentres], cy[kMaxGaussCentres], cz[kMaxGaussCentres];
};

// exp(-0.5 * (c * c) / (s * s))
__device__ __forceinline__ double gauss1(double c, double s) { return exp(dq(dm(-0.5, dm(c, c)), dm(s, s))); }

// DataInitializer::init_with_cos / init_with_gauss / init_with_multiple_gauss /
// init_with_setup_gauss (initializer.cpp:46-219): psi_0 on the interior
// 1..n-2 (the boundary stays zero), written as interleaved complex128.
__global__ void k_init_psi(double *__restrict__ psi, InitGeom g, const PsiCoef c) {
    const size_t N = (size_t)g.nx * g.ny * g.nz;
    const double twopi = 2. * 3.14159265358979323846; // 2 * M_PI, as the reference computes it
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N; q += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(q % g.nz);
        const int j = (int)((q / g.nz) % g.ny);
        const int i = (int)(q / ((size_t)g.nz * g.ny));
        double val  = 0.;
        if (i >= 1 && i < g.nx - 1 && j >= 1 && j < g.ny - 1 && k >= 1 && k < g.nz - 1) {
            const double X = coord(i, g.nx, g.dx), Y = coord(j, g.ny, g.dy), Z = coord(k, g.nz, g.dz);
            if (c.strategy == INIT_COS) {
                val = dm(dm(cos(dq(dm(twopi, ds(X, c.dd)), c.rrr)), cos(dq(dm(twopi, Y), c.rrr))),
                         cos(dq(dm(3.14159265358979323846, Z), c.rrr)));
            } else if (c.strategy == INIT_GAUSS) {
                val = dm(dm(gauss1(X, c.sx), gauss1(Y, c.sy)), gauss1(Z, c.sz));
            } else {
                for (int n = 0; n < c.ncent; ++n) {
                    const double xc = ds(X, c.cx[n]), yc = ds(Y, c.cy[n]);
                    const double zc = c.zcent ? ds(Z, c.cz[n]) : Z;
                    val = da(val, dm(dm(gauss1(xc, c.sx), gauss1(yc, c.sy)), gauss1(zc, c.sz)));
                }
            }
        }
        psi[2 * q]     = val;
        psi[2 * q + 1] = 0.;
    }
}

} // namespace gpe
