// Device kernels of the GPE solver path (templated on the working precision R).
//
// Field layout (device):
//   psi, psii, bnd : cplx<R>[nx*ny*nz], row-major (i*ny + j)*nz + k, z fastest
//   V, phi         : R[nx*ny*nz]
//   A              : cplx<R>[nx * 2ny * H], H = nz + 1, index (i*2ny + ky)*H + kz:
//                    the dipolar half spectrum with the x axis still in real
//                    space and pruned to the nx planes that are non-zero.
//
// The dipolar convolution of the reference (src/solver/fft_solvers/cpu/
// fftw_poisson_solver.cpp:51-96: zero-pad w|psi|^2 into (2nx,2ny,2nz), R2C,
// multiply by kz^2/k^2, C2R, keep the first octant, scale 1/(8N)) is evaluated
// exactly, but the transforms are pruned: the z pass reads only the nz non-zero
// samples of each padded line and writes the nz+1 kept bins; the y pass reads
// ny rows and writes 2ny; the x pass (forward, multiply, inverse fused in one
// kernel) reads nx planes and writes nx planes; the inverse passes keep only the
// first octant.
#pragma once

#include "fft_block.cuh"

namespace gpe {

// Per-iteration coefficients of the nonlinear phase (real-time half steps).
struct StepCoef {
    double g3w;  // (ggp11 - cdd/3) * n_atoms
    double gw15; // gamma * w_15
};

template <class R> __device__ __forceinline__ void sincos_r(R x, R *s, R *c);
template <> __device__ __forceinline__ void sincos_r<float>(float x, float *s, float *c) {
    sincosf(x, s, c);
}
template <> __device__ __forceinline__ void sincos_r<double>(double x, double *s, double *c) {
    sincos(x, s, c);
}

extern __shared__ __align__(16) unsigned char g_smem[];

// ---------------------------------------------------------------------------
// Dipolar convolution (Poisson::execute)
// ---------------------------------------------------------------------------

// z pass, forward: rho = w * s2 * |psi|^2 on the nz samples of each (i, j < ny)
// line, zero-padded to 2nz, complex FFT of length 2nz, keep the H = nz+1 bins.
// s2 = 1/xnorma when psi is held unnormalised (norm_state[0] = xnorma).
template <class R>
__global__ void __launch_bounds__(256)
    k_dip_z_fwd(const cplx<R> *__restrict__ psi, const double *__restrict__ norm_state, int lazy,
                cplx<R> *__restrict__ A, int nx, int ny, int nz, R w, LinePlan ln, int TB) {
    using C         = cplx<R>;
    const int TS    = TB + 1; // odd tile stride: the transposing loads hit distinct banks
    C *b0           = reinterpret_cast<C *>(g_smem);
    C *b1           = b0 + (size_t)TS * ln.L;
    const int H     = nz + 1;
    const int lines = nx * ny;
    const int l0    = blockIdx.x * TB;
    const int cnt   = min(TB, lines - l0);
    const R ws      = lazy ? (R)((double)w / norm_state[0]) : w;
    for (int e = threadIdx.x; e < cnt * nz; e += blockDim.x) {
        const int b = e / nz, k = e - b * nz;
        const C v   = psi[(size_t)(l0 + b) * nz + k];
        b0[k * TS + b] = C{(v.x * v.x + v.y * v.y) * ws, (R)0};
    }
    for (int e = threadIdx.x; e < cnt * (ln.L - nz); e += blockDim.x) {
        const int b = e % cnt, k = nz + e / cnt;
        b0[k * TS + b] = C{(R)0, (R)0};
    }
    __syncthreads();
    C *res = block_fft<-1, R>(b0, b1, ln, cnt, 1, TS, threadIdx.x, blockDim.x);
    for (int e = threadIdx.x; e < cnt * H; e += blockDim.x) {
        const int b = e / H, kz = e - b * H;
        const int l = l0 + b, i = l / ny, j = l - i * ny;
        A[((size_t)i * 2 * ny + j) * H + kz] = res[kz * TS + b];
    }
}

// y pass over one x plane, a tile of TB consecutive kz columns: n_in valid rows
// (the rest zero), transform of length L = 2ny, keep n_out rows.
template <int SIGN, class R>
__global__ void __launch_bounds__(256)
    k_dip_y(cplx<R> *__restrict__ A, int ny, int H, int n_in, int n_out, LinePlan ln, int TB) {
    using C        = cplx<R>;
    C *b0          = reinterpret_cast<C *>(g_smem);
    C *b1          = b0 + (size_t)TB * ln.L;
    const int i    = blockIdx.y;
    const int kz0  = blockIdx.x * TB;
    const int cnt  = min(TB, H - kz0);
    C *plane       = A + (size_t)i * 2 * ny * H;
    for (int e = threadIdx.x; e < cnt * n_in; e += blockDim.x) {
        const int j = e / cnt, b = e - j * cnt;
        b0[j * TB + b] = plane[(size_t)j * H + kz0 + b];
    }
    for (int e = threadIdx.x; e < cnt * (ln.L - n_in); e += blockDim.x) {
        const int j = n_in + e / cnt, b = e % cnt;
        b0[j * TB + b] = C{(R)0, (R)0};
    }
    __syncthreads();
    C *res = block_fft<SIGN, R>(b0, b1, ln, cnt, 1, TB, threadIdx.x, blockDim.x);
    for (int e = threadIdx.x; e < cnt * n_out; e += blockDim.x) {
        const int j = e / cnt, b = e - j * cnt;
        plane[(size_t)j * H + kz0 + b] = res[j * TB + b];
    }
}

// x pass: for TB consecutive (ky, kz) columns, forward FFT of length 2nx over the
// nx non-zero planes, multiply by V_dd(k) = kz^2/k^2 (reduced table indexed by
// |kx|, |ky|, kz) times dscale, inverse FFT, keep the first nx planes.
template <class R>
__global__ void __launch_bounds__(256)
    k_dip_x(cplx<R> *__restrict__ A, const R *__restrict__ vk, int nx, int ny, int H, R dscale,
            LinePlan ln, int TB) {
    using C         = cplx<R>;
    C *b0           = reinterpret_cast<C *>(g_smem);
    C *b1           = b0 + (size_t)TB * ln.L;
    const int cols  = 2 * ny * H;
    const int c0    = blockIdx.x * TB;
    const int cnt   = min(TB, cols - c0);
    const size_t ps = (size_t)cols; // plane stride
    for (int e = threadIdx.x; e < cnt * nx; e += blockDim.x) {
        const int i = e / cnt, b = e - i * cnt;
        b0[i * TB + b] = A[(size_t)i * ps + c0 + b];
    }
    for (int e = threadIdx.x; e < cnt * nx; e += blockDim.x) {
        const int i = nx + e / cnt, b = e % cnt;
        b0[i * TB + b] = C{(R)0, (R)0};
    }
    __syncthreads();
    C *res        = block_fft<-1, R>(b0, b1, ln, cnt, 1, TB, threadIdx.x, blockDim.x);
    C *other      = (res == b0) ? b1 : b0;
    const int L   = ln.L; // 2nx
    for (int e = threadIdx.x; e < cnt * L; e += blockDim.x) {
        const int t = e / cnt, b = e - t * cnt;
        const int c = c0 + b, ky = c / H, kz = c - ky * H;
        const int ix = t <= nx ? t : L - t;
        const int iy = ky <= ny ? ky : 2 * ny - ky;
        const R v    = vk[((size_t)ix * (ny + 1) + iy) * H + kz] * dscale;
        res[t * TB + b] = cscale(res[t * TB + b], v);
    }
    __syncthreads();
    C *res2 = block_fft<+1, R>(res, other, ln, cnt, 1, TB, threadIdx.x, blockDim.x);
    for (int e = threadIdx.x; e < cnt * nx; e += blockDim.x) {
        const int i = e / cnt, b = e - i * cnt;
        A[(size_t)i * ps + c0 + b] = res2[i * TB + b];
    }
}

// z pass, inverse (C2R): the H kept bins of each (i, j < ny) line, Hermitian-
// extended to 2nz, complex inverse FFT, real part of the first nz samples times
// inv_n (1/(8N)) -> phi.
template <class R>
__global__ void __launch_bounds__(256)
    k_dip_z_inv(const cplx<R> *__restrict__ A, R *__restrict__ phi, int nx, int ny, int nz, R inv_n,
                LinePlan ln, int TB) {
    using C         = cplx<R>;
    const int TS    = TB + 1;
    C *b0           = reinterpret_cast<C *>(g_smem);
    C *b1           = b0 + (size_t)TS * ln.L;
    const int H     = nz + 1;
    const int L     = ln.L; // 2nz
    const int lines = nx * ny;
    const int l0    = blockIdx.x * TB;
    const int cnt   = min(TB, lines - l0);
    for (int e = threadIdx.x; e < cnt * L; e += blockDim.x) {
        const int b = e / L, m = e - b * L;
        const int l = l0 + b, i = l / ny, j = l - i * ny;
        const C *line = A + ((size_t)i * 2 * ny + j) * H;
        C v;
        if (m < H) {
            v = line[m];
        } else {
            const C u = line[L - m];
            v         = C{u.x, -u.y};
        }
        b0[m * TS + b] = v;
    }
    __syncthreads();
    C *res = block_fft<+1, R>(b0, b1, ln, cnt, 1, TS, threadIdx.x, blockDim.x);
    for (int e = threadIdx.x; e < cnt * nz; e += blockDim.x) {
        const int b = e / nz, k = e - b * nz;
        phi[(size_t)(l0 + b) * nz + k] = res[k * TS + b].x * inv_n;
    }
}

// ---------------------------------------------------------------------------
// Kinetic step (Split::execute): 3D C2C FFT of psi, multiply by
// exp(i (-dt/2m) k^2) / N, inverse 3D FFT -- in place on psi.
// ---------------------------------------------------------------------------

// z lines (contiguous), TB lines per CTA.
template <int SIGN, class R>
__global__ void __launch_bounds__(256)
    k_kin_z(cplx<R> *__restrict__ psi, int lines, int nz, LinePlan ln, int TB) {
    using C       = cplx<R>;
    const int TS  = TB + 1;
    C *b0         = reinterpret_cast<C *>(g_smem);
    C *b1         = b0 + (size_t)TS * ln.L;
    const int l0  = blockIdx.x * TB;
    const int cnt = min(TB, lines - l0);
    C *base       = psi + (size_t)l0 * nz;
    for (int e = threadIdx.x; e < cnt * nz; e += blockDim.x) {
        const int b = e / nz, k = e - b * nz;
        b0[k * TS + b] = base[e];
    }
    __syncthreads();
    C *res = block_fft<SIGN, R>(b0, b1, ln, cnt, 1, TS, threadIdx.x, blockDim.x);
    for (int e = threadIdx.x; e < cnt * nz; e += blockDim.x) {
        const int b = e / nz, k = e - b * nz;
        base[e]     = res[k * TS + b];
    }
}

// y lines of one x plane, tile of TB consecutive k.
template <int SIGN, class R>
__global__ void __launch_bounds__(256)
    k_kin_y(cplx<R> *__restrict__ psi, int ny, int nz, LinePlan ln, int TB) {
    using C       = cplx<R>;
    C *b0         = reinterpret_cast<C *>(g_smem);
    C *b1         = b0 + (size_t)TB * ln.L;
    const int i   = blockIdx.y;
    const int k0  = blockIdx.x * TB;
    const int cnt = min(TB, nz - k0);
    C *plane      = psi + (size_t)i * ny * nz;
    for (int e = threadIdx.x; e < cnt * ny; e += blockDim.x) {
        const int j = e / cnt, b = e - j * cnt;
        b0[j * TB + b] = plane[(size_t)j * nz + k0 + b];
    }
    __syncthreads();
    C *res = block_fft<SIGN, R>(b0, b1, ln, cnt, 1, TB, threadIdx.x, blockDim.x);
    for (int e = threadIdx.x; e < cnt * ny; e += blockDim.x) {
        const int j = e / cnt, b = e - j * cnt;
        plane[(size_t)j * nz + k0 + b] = res[j * TB + b];
    }
}

// Unit-modulus factor applied as v + v*w with w = exp(i theta) - 1 given to
// full relative precision: the factor's modulus error is then ~eps*theta^2
// instead of ~eps, so repeated application does not bias the norm.
template <class C> __device__ __forceinline__ C apply_wm1(C v, C w) {
    return C{v.x + (v.x * w.x - v.y * w.y), v.y + (v.x * w.y + v.y * w.x)};
}
// (1+a)(1+b)(1+c) - 1 for small a, b, c
template <class C> __device__ __forceinline__ C combine_wm1(C a, C b, C c) {
    const C ab = cadd(cadd(a, b), cmul(a, b));
    return cadd(cadd(ab, c), cmul(ab, c));
}

// x lines for TB consecutive (j, k) columns: forward FFT, multiply by the
// kinetic phase exp(i(-dt/2m)(kx^2 + ky^2 + kz^2)) built from per-axis tables of
// exp(i theta) - 1 (FP64-computed), scale by 1/N = inv_hi + inv_lo, inverse.
template <class R>
__global__ void __launch_bounds__(256)
    k_kin_x(cplx<R> *__restrict__ psi, const cplx<R> *__restrict__ ex, const cplx<R> *__restrict__ ey,
            const cplx<R> *__restrict__ ez, R inv_hi, R inv_lo, int nx, int ny, int nz, LinePlan ln,
            int TB) {
    using C         = cplx<R>;
    C *b0           = reinterpret_cast<C *>(g_smem);
    C *b1           = b0 + (size_t)TB * ln.L;
    const int cols  = ny * nz;
    const int c0    = blockIdx.x * TB;
    const int cnt   = min(TB, cols - c0);
    for (int e = threadIdx.x; e < cnt * nx; e += blockDim.x) {
        const int i = e / cnt, b = e - i * cnt;
        b0[i * TB + b] = psi[(size_t)i * cols + c0 + b];
    }
    __syncthreads();
    C *res   = block_fft<-1, R>(b0, b1, ln, cnt, 1, TB, threadIdx.x, blockDim.x);
    C *other = (res == b0) ? b1 : b0;
    for (int e = threadIdx.x; e < cnt * nx; e += blockDim.x) {
        const int i = e / cnt, b = e - i * cnt;
        const int c = c0 + b, j = c / nz, k = c - j * nz;
        const C w   = combine_wm1(__ldg(&ex[i]), __ldg(&ey[j]), __ldg(&ez[k]));
        const C v   = apply_wm1(res[i * TB + b], w);
        res[i * TB + b] = C{fma(v.x, inv_hi, v.x * inv_lo), fma(v.y, inv_hi, v.y * inv_lo)};
    }
    __syncthreads();
    C *res2 = block_fft<+1, R>(res, other, ln, cnt, 1, TB, threadIdx.x, blockDim.x);
    for (int e = threadIdx.x; e < cnt * nx; e += blockDim.x) {
        const int i = e / cnt, b = e - i * cnt;
        psi[(size_t)i * cols + c0 + b] = res2[i * TB + b];
    }
}

// ---------------------------------------------------------------------------
// Real-time potential half step (cpu_solver.cpp:99-131): interior 1..n-2 only.
// psi *= exp(-i dt/2 (V + cdd phi + g3w |psi|^2 + gw15 |psi|^3)).
// The coefficients of iteration (*iter_base + local) come from coef[].
// ---------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(256)
    k_phase(cplx<R> *__restrict__ psi, const R *__restrict__ V, const R *__restrict__ phi,
            const StepCoef *__restrict__ coef, const int *__restrict__ iter_base, int local, int nx,
            int ny, int nz, R half_dt, R cdd) {
    using C             = cplx<R>;
    const StepCoef cf   = coef[*iter_base + local];
    const R g3w         = (R)cf.g3w, gw15 = (R)cf.gw15;
    const size_t N      = (size_t)nx * ny * nz;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N;
         q += (size_t)gridDim.x * blockDim.x) {
        const int k  = (int)(q % nz);
        const int j  = (int)((q / nz) % ny);
        const int i  = (int)(q / ((size_t)nz * ny));
        if (i < 1 || i >= nx - 1 || j < 1 || j >= ny - 1 || k < 1 || k >= nz - 1)
            continue;
        const C p       = psi[q];
        const R dens    = p.x * p.x + p.y * p.y;
        const R a       = sqrt(dens);
        const R v_int   = g3w * dens + gw15 * (a * a * a);
        const R total   = V[q] + cdd * phi[q] + v_int;
        // exp(i theta) - 1 = (-2 sin^2(theta/2), sin(theta)), theta = -dt/2 * total
        R s, c;
        sincos_r<R>((R)-0.5 * half_dt * total, &s, &c);
        const C w = C{(R)-2 * s * s, (R)2 * s * c};
        psi[q]    = apply_wm1(p, w);
    }
}

// ---------------------------------------------------------------------------
// Imaginary-time Euler update (cpu_solver.cpp:50-97), fused linear + nonlinear:
//   psi' = psi - dtau [ cx (psi_{i-1} + psi_{i+1} - 2psi) - cy (...) - cz (...)
//                       + (V + cdd phi) psi + (g3w |psi|^2 + gw15 |psi|^3) psi ]
// with psi = psi_in / sqrt(divisor[0]) (the pending normalisation), interior only; the
// boundary of psi' takes the values last loaded (the reference's cpsii keeps
// them).  Each block writes the FP64 partial sum of |psi'|^2 over its cells.
// ---------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(256)
    k_it_update(const cplx<R> *__restrict__ pin, cplx<R> *__restrict__ pout,
                const cplx<R> *__restrict__ bnd, const R *__restrict__ V, const R *__restrict__ phi,
                const double *__restrict__ divisor, const StepCoef *__restrict__ coef,
                double *__restrict__ partial, int nx, int ny, int nz, R cx, R cy, R cz, R dtau,
                R cdd) {
    using C        = cplx<R>;
    const R s      = (R)(1.0 / sqrt(divisor[0]));
    const R g3w    = (R)coef->g3w, gw15 = (R)coef->gw15;
    const size_t N = (size_t)nx * ny * nz;
    const size_t plane = (size_t)ny * nz;
    double acc     = 0.0;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N;
         q += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(q % nz);
        const int j = (int)((q / nz) % ny);
        const int i = (int)(q / plane);
        C o;
        if (i < 1 || i >= nx - 1 || j < 1 || j >= ny - 1 || k < 1 || k >= nz - 1) {
            o = bnd[q];
        } else {
            const C c0 = cscale(pin[q], s);
            const C xm = cscale(pin[q - plane], s), xp = cscale(pin[q + plane], s);
            const C ym = cscale(pin[q - nz], s), yp = cscale(pin[q + nz], s);
            const C zm = cscale(pin[q - 1], s), zp = cscale(pin[q + 1], s);
            const R vv   = V[q] + cdd * phi[q];
            const R dens = c0.x * c0.x + c0.y * c0.y;
            const R a    = sqrt(dens);
            const R nl   = g3w * dens + gw15 * (a * a * a);
            const R lr   = cx * ((xm.x + xp.x) - 2 * c0.x) - cy * ((ym.x + yp.x) - 2 * c0.x) -
                         cz * ((zm.x + zp.x) - 2 * c0.x) + c0.x * vv + nl * c0.x;
            const R li = cx * ((xm.y + xp.y) - 2 * c0.y) - cy * ((ym.y + yp.y) - 2 * c0.y) -
                         cz * ((zm.y + zp.y) - 2 * c0.y) + c0.y * vv + nl * c0.y;
            o = C{c0.x - dtau * lr, c0.y - dtau * li};
        }
        pout[q] = o;
        acc += (double)o.x * o.x + (double)o.y * o.y;
    }
    // block reduction in a fixed order
    __shared__ double red[32];
    for (int off = 16; off > 0; off >>= 1)
        acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int off = 16; off > 0; off >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, off);
        if (threadIdx.x == 0)
            partial[blockIdx.x] = v;
    }
}

// Sum of |psi|^2 per block (FP64), with the lazy scale applied.
template <class R>
__global__ void __launch_bounds__(256)
    k_norm_partial(const cplx<R> *__restrict__ psi, size_t N, double *__restrict__ partial) {
    double acc = 0.0;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N;
         q += (size_t)gridDim.x * blockDim.x) {
        const cplx<R> p = psi[q];
        acc += (double)p.x * p.x + (double)p.y * p.y;
    }
    __shared__ double red[32];
    for (int off = 16; off > 0; off >>= 1)
        acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int off = 16; off > 0; off >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, off);
        if (threadIdx.x == 0)
            partial[blockIdx.x] = v;
    }
}

// norm_state[0] = xnorma = dV * sum(partial) (fixed order; one block of 256).
// norm_state[1] = 1 / sqrt(xnorma).  status[0] is set to 1 on a non-finite norm.
__global__ void __launch_bounds__(256)
    k_norm_finalize(const double *__restrict__ partial, int nparts, double dV,
                    double *__restrict__ norm_state, int *__restrict__ status);

// psi *= 1/sqrt(norm_state[0]) (materialise the lazy normalisation).
template <class R>
__global__ void __launch_bounds__(256)
    k_scale(cplx<R> *__restrict__ psi, size_t N, const double *__restrict__ norm_state) {
    const R s = (R)(1.0 / sqrt(norm_state[0]));
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N;
         q += (size_t)gridDim.x * blockDim.x)
        psi[q] = cscale(psi[q], s);
}

// ---------------------------------------------------------------------------
// Energies (cpu_solver.cpp:137-194): per-block FP64 partials of the five sums
// over the interior; partial layout [5][nblocks].
// ---------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(256)
    k_energy_partial(const cplx<R> *__restrict__ pin, const R *__restrict__ V,
                     const R *__restrict__ phi, const double *__restrict__ norm_state, int lazy,
                     double *__restrict__ partial, int nx, int ny, int nz, double idx2, double idy2,
                     double idz2, double ggp11, double cdd, double n_atoms, double gamma) {
    const double s     = lazy ? 1.0 / sqrt(norm_state[0]) : 1.0;
    const size_t N     = (size_t)nx * ny * nz;
    const size_t plane = (size_t)ny * nz;
    double e[5]        = {0, 0, 0, 0, 0};
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N;
         q += (size_t)gridDim.x * blockDim.x) {
        // grids hold at most 2^30 points: 32-bit index arithmetic
        const unsigned q32 = (unsigned)q, row = q32 / (unsigned)nz;
        const int k = (int)(q32 - row * (unsigned)nz);
        const int i = (int)(row / (unsigned)ny);
        const int j = (int)(row - (unsigned)i * (unsigned)ny);
        if (i < 1 || i >= nx - 1 || j < 1 || j >= ny - 1 || k < 1 || k >= nz - 1)
            continue;
        auto ld = [&](size_t t) {
            const cplx<R> v = pin[t];
            return double2{(double)v.x * s, (double)v.y * s};
        };
        const double2 c0 = ld(q), xm = ld(q - plane), xp = ld(q + plane), ym = ld(q - nz),
                      yp = ld(q + nz), zm = ld(q - 1), zp = ld(q + 1);
        const double gr = -((xp.x + xm.x) - 2. * c0.x) * idx2 - ((yp.x + ym.x) - 2. * c0.x) * idy2 -
                          ((zp.x + zm.x) - 2. * c0.x) * idz2;
        const double gi = -((xp.y + xm.y) - 2. * c0.y) * idx2 - ((yp.y + ym.y) - 2. * c0.y) * idy2 -
                          ((zp.y + zm.y) - 2. * c0.y) * idz2;
        const double nrm = c0.x * c0.x + c0.y * c0.y;
        e[0] += gr * c0.x + gi * c0.y;
        e[1] += (double)V[q] * nrm;
        e[2] += 0.5 * ggp11 * nrm * nrm;
        e[3] += 0.5 * cdd * (double)phi[q] * nrm * n_atoms -
                cdd / 3. * (nrm * nrm) / 2. * (n_atoms * n_atoms);
        e[4] += 2. / 5. * gamma * (nrm * nrm * sqrt(nrm));
    }
    __shared__ double red[5][32];
#pragma unroll
    for (int t = 0; t < 5; ++t) {
        double v = e[t];
        for (int off = 16; off > 0; off >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0)
            red[t][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int t = 0; t < 5; ++t) {
            double v = threadIdx.x < (blockDim.x >> 5) ? red[t][threadIdx.x] : 0.0;
            for (int off = 16; off > 0; off >>= 1)
                v += __shfl_down_sync(0xffffffffu, v, off);
            if (threadIdx.x == 0)
                partial[(size_t)t * gridDim.x + blockIdx.x] = v;
        }
    }
}

// out[t] = sum over blocks of partial[t][*] (t < 5), fixed order.
__global__ void __launch_bounds__(256)
    k_energy_finalize(const double *__restrict__ partial, int nparts, double *__restrict__ out);

// ---------------------------------------------------------------------------
// Host-format conversion: FP64 staging <-> working precision.
// ---------------------------------------------------------------------------
template <class R>
__global__ void k_from_f64(const double *__restrict__ src, R *__restrict__ dst, size_t n) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
         q += (size_t)gridDim.x * blockDim.x)
        dst[q] = (R)src[q];
}

// dst = scale * src (scale = 1/sqrt(norm_state[0]) when lazy), widened to FP64.
template <class R>
__global__ void k_to_f64(const R *__restrict__ src, double *__restrict__ dst, size_t n,
                         const double *__restrict__ norm_state, int lazy) {
    const double s = lazy ? 1.0 / sqrt(norm_state[0]) : 1.0;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
         q += (size_t)gridDim.x * blockDim.x)
        dst[q] = (double)src[q] * s;
}

__global__ void k_advance(int *counter, int by);

} // namespace gpe
