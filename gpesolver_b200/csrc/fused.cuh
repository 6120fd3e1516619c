// Fused iteration pipeline (compile-time line lengths).
//
// One imaginary- or real-time iteration is four kernels, each a batch of 1D
// FFT lines along one axis with the elementwise physics fused into its loads
// and stores:
//
//   X  pencils along x: kinetic  fwd FFT(nx) * (exp(i(-dt/2m)k^2) - 1)/N * inv FFT(nx)
//                       dipolar  fwd FFT(2nx, upper half zero) * V_dd(k) * scale
//                                * inv FFT(2nx), first nx kept
//   Yi lines along y, inverse:   kinetic iFFT(ny); dipolar iFFT(2ny), first ny kept
//   Z  rows along z:   dipolar C2R (pairs of rows packed in one complex FFT of
//                      2nz) -> phi; kinetic iFFT(nz) -> the kinetic increment,
//                      added to the kept real-space psi (psi_r); the real-time phases
//                      of two consecutive half steps merged into one rotation
//                      (they see the same |psi|, V and phi); rho = w|psi|^2;
//                      kinetic FFT(nz); dipolar R2C (pairs) -> spectrum
//                      (imaginary time: the Euler stencil update instead of the
//                      kinetic transforms, with the norm reduced on the fly)
//   Yf lines along y, forward:   kinetic FFT(ny); dipolar FFT(2ny, upper half zero)
//
// Dipolar spectrum layout: S[i][ky][kz-1], i < nx (x in real space between the
// X passes), ky < 2ny, 1 <= kz <= nz.  The kz = 0 plane is not stored: V_dd is
// kz^2/k^2, exactly 0 on that plane (fftw_poisson_solver.cpp:39-45), so it adds
// nothing to phi.
#pragma once

#include "ct_fft.cuh"
#include "kernels.cuh"
#include "rfft.cuh"

namespace gpe {

// Tile widths (lines per CTA) for a pass of line length L in precision R:
// CNT*L complex within 32 KiB (one in-place tile buffer per CTA).
template <class R, int L> constexpr int tile_lines() {
    int c = (int)(32768 / (int)sizeof(cplx<R>) / L);
    int p = 1;
    while (p * 2 <= c && p * 2 <= 32)
        p *= 2;
    return p;
}

struct Twid {
    const void *tw;
    const void *lo;
};

struct StepIdx {
    const StepCoef *coef; // per-iteration coefficients of this call
    const int *base;      // device counter: index of the chunk's first iteration
    int local;            // iteration within the chunk
};

enum { ZM_RT_PRO = 0, ZM_RT_MID, ZM_RT_EPI, ZM_IT_PRO, ZM_IT_MID };

// Asynchronous global -> shared copies (cp.async, completion per thread; a
// barrier after the wait makes the data visible to the block).
__device__ __forceinline__ void cp_async8(void *smem, const void *g) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *g) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// wait until at most N of this thread's committed groups are pending
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// One-dimensional bulk copies (global -> this CTA's shared memory) completing
// on an mbarrier: one thread arms the barrier with the byte count and issues
// the copies, every thread waits for the barrier's phase.  Addresses and sizes
// must be multiples of 16 bytes.  No multicast: each CTA copies into its own
// shared memory.
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
    // make the initialised barrier visible to the async proxy (the bulk copies)
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *smem, const void *g, unsigned bytes, unsigned long long *bar) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(s),
                 "l"(g), "r"(bytes), "r"(b)
                 : "memory");
}
// Waits for phase `parity` of the barrier, at most `tries` polls (each poll may
// suspend the thread for a while); false when it gave up.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, int tries) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    for (int t = 0; t < tries; ++t) {
        unsigned done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (done)
            return true;
    }
    return false;
}


// ---------------------------------------------------------------------------
// X pencils
// ---------------------------------------------------------------------------
// Lines per CTA of the x passes: 8 or 16 (64 / 128-byte row segments per x),
// picked per grid by the solver's autotuner (Solver::autotune_x).

// Kinetic x pencils, increment form: psi(x, ky, kz) -> FFT_x ->
// (exp(i(-dt/2m)k^2) - 1) / N -> iFFT_x, i.e. the change the kinetic step makes
// to psi, which the z / plane kernel adds to the real-space psi it kept from the
// previous phase step (ZArgs::psi_r).  In exact arithmetic this is the kinetic
// step itself; in FP32 the rounding of the transforms scales with |e^{i theta} -
// 1| instead of with |psi|, so the per-step error is about one rounding of the
// sum instead of that of a forward and an inverse 3D FFT.  The forward transform
// ends and the inverse one starts in registers, with the factor applied in
// between.
template <class R, int NX, int CNT, int NT>
__global__ void __launch_bounds__(NT)
    k3_x_kin(cplx<R> *__restrict__ psi, const cplx<R> *__restrict__ ex, const cplx<R> *__restrict__ ey,
             const cplx<R> *__restrict__ ez, R inv_hi, R inv_lo, int ny, int nz, Twid tk) {
    using C  = cplx<R>;
    using Fw = LinePass<-1, R, NX, CNT, CNT, NT, true, false>;
    using Iv = LinePass<+1, R, NX, CNT, CNT, NT, true, true>;
    static_assert(Fw::RL == Iv::R0 && Fw::ROUNDSL == Iv::ROUNDS0 && Fw::ITEMSL == Iv::ITEMS0,
                  "paired transforms share the register layout");
    const int tid  = threadIdx.x;
    C *buf         = reinterpret_cast<C *>(g_smem);
    const C *tw    = (const C *)tk.tw, *tl = (const C *)tk.lo;
    const int cols = ny * nz;
    const int c0   = blockIdx.x * CNT;
    const int cnt  = min(CNT, cols - c0);
    // the line's (1+wy)(1+wz) - 1, read before the transform so that its L2
    // reads land behind the line loads
    const int b = Fw::line_of(tid);
    C wyz       = C{(R)0, (R)0};
    if (b < cnt) {
        const int c = c0 + b, j = c / nz, k = c - j * nz;
        const C wy = __ldg(&ey[j]), wz = __ldg(&ez[k]);
        wyz        = cadd(cadd(wy, wz), cmul(wy, wz));
    }
    C a[Fw::ROUNDSL][Fw::RL];
    Fw::run_to_regs(
        buf, [&](int b, int t) { return b < cnt ? psi[(size_t)t * cols + c0 + b] : C{(R)0, (R)0}; }, a, tw, tl,
        tid);
    {
#pragma unroll
        for (int rd = 0; rd < Fw::ROUNDSL; ++rd) {
            if (!Fw::template valid<Fw::ITEMSL>(rd * NT + tid))
                break;
#pragma unroll
            for (int q = 0; q < Fw::RL; ++q) {
                const C wx = __ldg(&ex[Fw::last_index(tid, rd, q)]);
                const C w  = cadd(cadd(wx, wyz), cmul(wx, wyz)); // (1+wx)(1+wyz) - 1
                const C v  = cmul(a[rd][q], w);
                a[rd][q]   = C{fma(v.x, inv_hi, v.x * inv_lo), fma(v.y, inv_hi, v.y * inv_lo)};
            }
        }
    }
    __syncthreads();
    Iv::run_from_regs(
        buf, a,
        [&](int b, int t, C v) {
            if (b < cnt)
                psi[(size_t)t * cols + c0 + b] = v;
        },
        tw, tl, tid);
}

// Dipolar x pencils: S(x, ky, kz) -> FFT_2nx (upper half zero) -> V_dd(k) * scale
// -> iFFT_2nx, lower half kept.  scale = 1/(8N) (C2R normalisation) and, in
// imaginary time, 1/xnorma (the spectrum was built from the unnormalised psi).
// The twiddle table and the V_dd(k) values of the CTA's lines (|kx| = 0..nx) are
// copied into shared memory (cp.async) at kernel start, behind the forward
// transform's global loads, instead of being gathered from L2 after it.
template <class R, int NX, int CNT> constexpr size_t x_dip_smem() {
    return sizeof(cplx<R>) * (CNT * 2 * NX + 2 * NX) + sizeof(R) * (NX + 1) * CNT;
}

template <class R, int NX, int CNT, int NT>
__global__ void __launch_bounds__(NT, NX >= 256 ? 2 : 3) // 512-point lines: two CTAs per SM; 256: three
    k3_x_dip(cplx<R> *__restrict__ S, const R *__restrict__ vk, const double *__restrict__ divisor,
             double dip_scale, int ny, int nz, Twid td) {
    using C          = cplx<R>;
    constexpr int L  = 2 * NX;
    // two-stage lines (radix pairs) take their twiddles from the shared copy;
    // longer radix chains (nx = 96) keep the global table in the middle stages
    constexpr bool TW2 = radices_of(L).n == 2;
    using Fw         = LinePass<-1, R, L, CNT, CNT, NT, false, false, true, false, TW2>;
    using Iv         = LinePass<+1, R, L, CNT, CNT, NT, false, true, false, true, TW2>;
    static_assert(Fw::RL == Iv::R0 && Fw::ROUNDSL == Iv::ROUNDS0 && Fw::ITEMSL == Iv::ITEMS0,
                  "paired transforms share the register layout");
    const int tid  = threadIdx.x;
    C *buf         = reinterpret_cast<C *>(g_smem);
    C *tws         = buf + CNT * L;                    // twiddles exp(-2 pi i m / L)
    R *vs          = reinterpret_cast<R *>(tws + L);   // V_dd of |kx| = 0..NX, line b: vs[|kx| CNT + b]
    const C *tw    = (const C *)td.tw;
    const C *twu   = TW2 ? tws : tw;                   // the table the stages read
    const int cols = 2 * ny * nz;
    const int c0   = blockIdx.x * CNT;
    const int cnt  = min(CNT, cols - c0);
    const size_t xs = (size_t)(ny + 1) * nz;
    for (int m = tid; m < L; m += NT)
        cp_async8(&tws[m], &tw[m]);
    for (int e = tid; e < (NX + 1) * CNT; e += NT) {
        const int ix = e / CNT, b = e - ix * CNT;
        const int c  = min(c0 + b, cols - 1);
        const int ky = c / nz, kz = c - ky * nz;
        const int iy = ky <= ny ? ky : 2 * ny - ky;
        cp_async4(&vs[e], &vk[(size_t)ix * xs + (size_t)iy * nz + kz]);
    }
    cp_async_commit();
    // the spectrum's scale (imaginary time: over the norm of the psi it was
    // built from), read before the transform
    const R scale = (R)(divisor ? dip_scale / divisor[0] : dip_scale);
    auto ld = [&](int b, int t) { return b < cnt ? S[(size_t)t * cols + c0 + b] : C{(R)0, (R)0}; };
    C a[Fw::ROUNDSL][Fw::RL];
    Fw::stage0_to_tile(buf, ld, tid);
    cp_async_wait<0>();
    __syncthreads();
    Fw::template middle<1>(buf, twu, nullptr, tid);
#pragma unroll
    for (int rd = 0; rd < Fw::ROUNDSL; ++rd) {
        const int it = rd * NT + tid;
        if (!Fw::template valid<Fw::ITEMSL>(it))
            break;
        const int j = it / CNT, b = it - j * CNT;
        Fw::loadL(buf, a[rd], j, b, twu, nullptr);
    }
    {
        const int b   = Fw::line_of(tid);
#pragma unroll
        for (int rd = 0; rd < Fw::ROUNDSL; ++rd) {
            if (!Fw::template valid<Fw::ITEMSL>(rd * NT + tid))
                break;
#pragma unroll
            for (int q = 0; q < Fw::RL; ++q) {
                const int t  = Fw::last_index(tid, rd, q);
                const int ix = t <= NX ? t : L - t;
                a[rd][q]     = cscale(a[rd][q], vs[ix * CNT + b] * scale);
            }
        }
    }
    __syncthreads();
    Iv::run_from_regs(
        buf, a,
        [&](int b, int t, C v) {
            if (b < cnt)
                S[(size_t)t * cols + c0 + b] = v;
        },
        twu, nullptr, tid);
}

// ---------------------------------------------------------------------------
// Y lines (one x plane per blockIdx.y; z-column tiles along blockIdx.x)
// ---------------------------------------------------------------------------
template <class R, int NY, int SIGN, int CNT, int NT>
__global__ void __launch_bounds__(NT) k3_y_kin(cplx<R> *__restrict__ psi, int nz, Twid tk) {
    using C       = cplx<R>;
    using P       = LinePass<SIGN, R, NY, CNT, CNT, NT, true, false>;
    const int k0  = blockIdx.x * CNT;
    const int cnt = min(CNT, nz - k0);
    C *plane      = psi + (size_t)blockIdx.y * NY * nz + k0;
    P::run(
        reinterpret_cast<C *>(g_smem),
        [&](int b, int t) { return b < cnt ? plane[(size_t)t * nz + b] : C{(R)0, (R)0}; },
        [&](int b, int t, C v) {
            if (b < cnt)
                plane[(size_t)t * nz + b] = v;
        },
        (const C *)tk.tw, (const C *)tk.lo, threadIdx.x);
}

// Dipolar y lines of length 2ny: forward (SIGN < 0) with the upper half of the
// input zero, inverse (SIGN > 0) with only the lower half of the output kept.
template <class R, int NY, int SIGN, int CNT, int NT>
__global__ void __launch_bounds__(NT) k3_y_dip(cplx<R> *__restrict__ S, int nz, Twid td) {
    using C         = cplx<R>;
    constexpr int L = 2 * NY;
    using P         = LinePass<SIGN, R, L, CNT, CNT, NT, false, (SIGN > 0), (SIGN < 0), (SIGN > 0)>;
    const int k0    = blockIdx.x * CNT;
    const int cnt   = min(CNT, nz - k0);
    C *plane        = S + (size_t)blockIdx.y * L * nz + k0;
    P::run(
        reinterpret_cast<C *>(g_smem),
        [&](int b, int t) { return b < cnt ? plane[(size_t)t * nz + b] : C{(R)0, (R)0}; },
        [&](int b, int t, C v) {
            if (b < cnt)
                plane[(size_t)t * nz + b] = v;
        },
        (const C *)td.tw, (const C *)td.lo, threadIdx.x);
}

// Shared memory of the x / y passes (one tile of COUNT lines).
template <class R, int L, int CNT> constexpr size_t xy_smem() { return sizeof(cplx<R>) * CNT * L; }

// y pass for ny = N with CNT z columns per tile.
template <class R, int N, int CNT> struct YShape {
    static constexpr int NTK = pass_threads<N, CNT>(), NTD = pass_threads<2 * N, CNT>();
    static constexpr size_t SK = xy_smem<R, N, CNT>(), SD = xy_smem<R, 2 * N, CNT>();
};

// ---------------------------------------------------------------------------
// Z rows
// ---------------------------------------------------------------------------
struct ZArgs {
    // fields
    void *psi_in;        // RT: the kinetic increment's yz spectrum (psi in RT_PRO); IT: psi
    void *psi_out;       // RT: same as psi_in; IT: the next psi buffer
    void *psi_r;         // RT: psi in real space after the last phase step (read, then rewritten)
    const void *bnd;     // IT: boundary values (last loaded psi)
    void *S;             // dipolar spectrum
    const void *V;
    void *phi;
    // norms (IT)
    double *norm_state;  // [0] xnorma, [1] divisor of psi_in (read), both written by the last CTA
    double *partial;     // per-CTA partial sums of |psi_out|^2
    unsigned *ticket;    // CTA completion counter (reset by the last CTA)
    int *status;
    double dV;
    // coefficients
    StepIdx step;
    double half_dt, cdd, w_atoms;
    double cx, cy, cz, dtau; // IT stencil
    int nx, ny;
};

template <class R, int NZ, int MODE>
__global__ void __launch_bounds__(256, 4) k2_z(ZArgs a, Twid tk, Twid td) {
    using C          = cplx<R>;
    constexpr int NT = 256;
    constexpr int RW = 32;          // rows per CTA
    constexpr int NP = RW / 2;      // row pairs for the real transforms
    constexpr int LD = 2 * NZ;      // dipolar line length
    constexpr int TK = RW + 1;      // tile strides (odd: transposing loads avoid bank conflicts)
    constexpr int TD = NP + 1;
    constexpr bool RT      = MODE <= ZM_RT_EPI;
    constexpr bool HAS_INV = (MODE == ZM_RT_MID || MODE == ZM_RT_EPI || MODE == ZM_IT_MID);
    constexpr bool HAS_FWD = (MODE != ZM_RT_EPI);
    const int tid          = threadIdx.x;
    const int nx = a.nx, ny = a.ny;
    const int rows = nx * ny;
    const int r0   = blockIdx.x * RW;

    C *kb0  = reinterpret_cast<C *>(g_smem); // kinetic tile [k][row]
    C *db0  = kb0 + TK * NZ;                 // dipolar pair tile [m][pair]
    R *phis = reinterpret_cast<R *>(db0 + TD * LD); // phi, then rho, [k][row]
    R *vs   = phis + TK * NZ;                // V tile [k][row] (real time)
    C *prs  = db0;                           // kept psi [row][k] (real time, after the C2R)
    __shared__ double red[8];

    const C *S_in = reinterpret_cast<const C *>(a.S);
    C *S_out      = reinterpret_cast<C *>(a.S);
    C *pr         = reinterpret_cast<C *>(a.psi_r);
    constexpr bool KEPT = MODE == ZM_RT_MID || MODE == ZM_RT_EPI;

    // real time: the kinetic tile and V are copied in (cp.async) behind the C2R
    if (RT) {
        const C *pin = reinterpret_cast<const C *>(a.psi_in);
        const R *Vg  = reinterpret_cast<const R *>(a.V);
        for (int e = tid; e < RW * NZ; e += NT) {
            const int row = e / NZ, k = e % NZ;
            const int rr  = r0 + row;
            if (rr < rows) {
                cp_async8(&kb0[row + k * TK], &pin[(size_t)rr * NZ + k]);
                cp_async4(&vs[row + k * TK], &Vg[(size_t)rr * NZ + k]);
            } else {
                kb0[row + k * TK] = C{(R)0, (R)0};
                vs[row + k * TK]  = (R)0;
            }
        }
        cp_async_commit();
    }

    // ---- phi: dipolar C2R of the row pairs -------------------------------
    if (HAS_INV) {
        // consecutive threads take consecutive m: the spectrum rows are read
        // contiguously (coalesced)
        for (int e = tid; e < NP * LD; e += NT) {
            const int m = e % LD, p = e / LD;
            const int ra = r0 + 2 * p, rb = ra + 1;
            C z = C{(R)0, (R)0};
            if (m > 0 && ra < rows) {
                const int ia = ra / ny, ja = ra - ia * ny;
                const int mm = m <= NZ ? m : LD - m;
                const C xa   = S_in[((size_t)ia * 2 * ny + ja) * NZ + (mm - 1)];
                C xb         = C{(R)0, (R)0};
                if (rb < rows) {
                    const int ib = rb / ny, jb = rb - ib * ny;
                    xb           = S_in[((size_t)ib * 2 * ny + jb) * NZ + (mm - 1)];
                }
                if (m == NZ)
                    z = C{xa.x, xb.x}; // self-conjugate bin: real parts only
                else if (m < NZ)
                    z = C{xa.x - xb.y, xa.y + xb.x};   // xa + i xb
                else
                    z = C{xa.x + xb.y, xb.x - xa.y};   // conj(xa) + i conj(xb)
            }
            db0[p + m * TD] = z;
        }
        __syncthreads();
        ct_fft_ip<+1, R, LD, NP, TD, NT, false, false, true>(db0, (const C *)td.tw, (const C *)td.lo, tid);
        const C *r = db0;
        R *phi_g = reinterpret_cast<R *>(a.phi);
        for (int e = tid; e < RW * NZ; e += NT) {
            const int row = e / NZ, k = e % NZ; // coalesced store along k
            const int p = row >> 1;
            const C zz  = r[p + k * TD];
            const R v   = (row & 1) ? zz.y : zz.x;
            phis[row + k * TK] = v;
            if (r0 + row < rows)
                phi_g[(size_t)(r0 + row) * NZ + k] = v;
        }
        __syncthreads();
        if (KEPT) {
            // the pair tile is free until the R2C: the kept psi goes there
            for (int e = tid; e < RW * NZ; e += NT) {
                const int row = e / NZ, k = e % NZ;
                const int rr  = r0 + row;
                if (rr < rows)
                    cp_async8(&prs[e], &pr[(size_t)rr * NZ + k]);
                else
                    prs[e] = C{(R)0, (R)0};
            }
            cp_async_commit();
        }
    } else if (RT) {
        // prologue: phi from the previous calc_fi3d
        const R *phi_g = reinterpret_cast<const R *>(a.phi);
        for (int e = tid; e < RW * NZ; e += NT) {
            const int row = e / NZ, k = e % NZ;
            phis[row + k * TK] = (r0 + row < rows) ? phi_g[(size_t)(r0 + row) * NZ + k] : (R)0;
        }
    }

    // ---- psi for the physics step -----------------------------------------
    C *kt = kb0; // tile holding psi in real space, [k][row]
    if (RT) {
        if (KEPT)
            cp_async_wait<1>(); // kinetic tile and V (the kept psi may still be in flight)
        else
            cp_async_wait<0>();
        __syncthreads();
        if (MODE != ZM_RT_PRO)
            ct_fft_ip<+1, R, NZ, RW, TK, NT>(kb0, (const C *)tk.tw, (const C *)tk.lo, tid);
    }

    double acc = 0.0;
    if (RT) {
        // merged potential half steps: theta = -dt/2 [cV (V + cdd phi) + g3 |psi|^2 + gw |psi|^3]
        R cV, g3, gw;
        {
            const int base = *a.step.base + a.step.local;
            const StepCoef c0 = a.step.coef[base];
            if (MODE == ZM_RT_MID) {
                const StepCoef c1 = a.step.coef[base + 1];
                cV = (R)2;
                g3 = (R)(c0.g3w + c1.g3w);
                gw = (R)(c0.gw15 + c1.gw15);
            } else {
                cV = (R)1;
                g3 = (R)c0.g3w;
                gw = (R)c0.gw15;
            }
        }
        const R hdt   = (R)a.half_dt, cdd = (R)a.cdd, wat = (R)a.w_atoms;
        if (KEPT) {
            cp_async_wait<0>();
            __syncthreads();
        }
        for (int e = tid; e < RW * NZ; e += NT) {
            const int row = e / NZ, k = e % NZ;
            const int rr  = r0 + row;
            if (rr >= rows)
                continue;
            const int i = rr / ny, j = rr - i * ny;
            C p         = kt[row + k * TK];
            if (MODE != ZM_RT_PRO)
                p = cadd(p, prs[e]); // psi + kinetic increment
            if (i >= 1 && i < nx - 1 && j >= 1 && j < ny - 1 && k >= 1 && k < NZ - 1) {
                const R dens  = p.x * p.x + p.y * p.y;
                const R am    = sqrt(dens);
                const R total = cV * (vs[row + k * TK] + cdd * phis[row + k * TK]) + g3 * dens +
                                gw * (am * am * am);
                R s, c;
                sincos_r<R>((R)-0.5 * hdt * total, &s, &c);
                p = apply_wm1(p, C{(R)-2 * s * s, (R)2 * s * c});
            }
            kt[row + k * TK] = p;
            if (MODE != ZM_RT_EPI)
                pr[(size_t)rr * NZ + k] = p;
            // rho for the next dipolar spectrum (stored in the phi tile)
            phis[row + k * TK] = wat * (p.x * p.x + p.y * p.y);
        }
        __syncthreads();
        if (MODE == ZM_RT_EPI) {
            C *pout = reinterpret_cast<C *>(a.psi_out);
            for (int e = tid; e < RW * NZ; e += NT) {
                const int row = e / NZ, k = e % NZ;
                if (r0 + row < rows)
                    pout[(size_t)(r0 + row) * NZ + k] = kt[row + k * TK];
            }
            return;
        }
        // kinetic forward z
        ct_fft_ip<-1, R, NZ, RW, TK, NT>(kb0, (const C *)tk.tw, (const C *)tk.lo, tid);
        const C *kf = kb0;
        C *pout     = reinterpret_cast<C *>(a.psi_out);
        for (int e = tid; e < RW * NZ; e += NT) {
            const int row = e / NZ, k = e % NZ;
            if (r0 + row < rows)
                pout[(size_t)(r0 + row) * NZ + k] = kf[row + k * TK];
        }
    } else {
        // imaginary time: psi_in / sqrt(divisor)
        const C *pin  = reinterpret_cast<const C *>(a.psi_in);
        C *pout       = reinterpret_cast<C *>(a.psi_out);
        const C *bnd  = reinterpret_cast<const C *>(a.bnd);
        const R sc    = (R)(1.0 / sqrt(a.norm_state[1]));
        const R wat   = (R)a.w_atoms;
        const size_t plane = (size_t)ny * NZ;
        if (MODE == ZM_IT_PRO) {
            for (int e = tid; e < RW * NZ; e += NT) {
                const int row = e / NZ, k = e % NZ;
                const int rr  = r0 + row;
                R rho         = (R)0;
                if (rr < rows) {
                    const C p = pin[(size_t)rr * NZ + k];
                    rho       = wat * (p.x * p.x + p.y * p.y);
                }
                phis[row + k * TK] = rho;
            }
        } else {
            const StepCoef cf = a.step.coef[0];
            const R g3w = (R)cf.g3w, gw15 = (R)cf.gw15;
            const R *Vg = reinterpret_cast<const R *>(a.V);
            const R cx = (R)a.cx, cy = (R)a.cy, cz = (R)a.cz, dtau = (R)a.dtau, cdd = (R)a.cdd;
            for (int e = tid; e < RW * NZ; e += NT) {
                const int row = e / NZ, k = e % NZ;
                const int rr  = r0 + row;
                R rho         = (R)0;
                if (rr < rows) {
                    const int i = rr / ny, j = rr - i * ny;
                    const size_t q = (size_t)rr * NZ + k;
                    C o;
                    if (i < 1 || i >= nx - 1 || j < 1 || j >= ny - 1 || k < 1 || k >= NZ - 1) {
                        o = bnd[q];
                    } else {
                        const C c0 = cscale(pin[q], sc);
                        const C xm = cscale(pin[q - plane], sc), xp = cscale(pin[q + plane], sc);
                        const C ym = cscale(pin[q - NZ], sc), yp = cscale(pin[q + NZ], sc);
                        const C zm = cscale(pin[q - 1], sc), zp = cscale(pin[q + 1], sc);
                        const R vv   = Vg[q] + cdd * phis[row + k * TK];
                        const R dens = c0.x * c0.x + c0.y * c0.y;
                        const R am   = sqrt(dens);
                        const R nl   = g3w * dens + gw15 * (am * am * am);
                        const R lr   = cx * ((xm.x + xp.x) - 2 * c0.x) - cy * ((ym.x + yp.x) - 2 * c0.x) -
                                     cz * ((zm.x + zp.x) - 2 * c0.x) + c0.x * vv + nl * c0.x;
                        const R li = cx * ((xm.y + xp.y) - 2 * c0.y) - cy * ((ym.y + yp.y) - 2 * c0.y) -
                                     cz * ((zm.y + zp.y) - 2 * c0.y) + c0.y * vv + nl * c0.y;
                        o = C{c0.x - dtau * lr, c0.y - dtau * li};
                    }
                    pout[q] = o;
                    acc += (double)o.x * o.x + (double)o.y * o.y;
                    rho = wat * (o.x * o.x + o.y * o.y);
                }
                phis[row + k * TK] = rho;
            }
        }
        __syncthreads();
    }

    // ---- dipolar R2C of rho (row pairs) -> spectrum -------------------------
    if (HAS_FWD) {
        // rows NZ..LD-1 are the zero padding (not read by the pruned first stage)
        for (int e = tid; e < NP * NZ; e += NT) {
            const int m = e % NZ, p = e / NZ;
            db0[p + m * TD] = C{phis[2 * p + m * TK], phis[2 * p + 1 + m * TK]};
        }
        __syncthreads();
        ct_fft_ip<-1, R, LD, NP, TD, NT, false, true, false>(db0, (const C *)td.tw, (const C *)td.lo, tid);
        const C *r = db0;
        for (int e = tid; e < RW * NZ; e += NT) {
            const int row = e / NZ, m = e % NZ + 1; // bins 1..NZ
            const int rr  = r0 + row;
            if (rr >= rows)
                continue;
            const int p  = row >> 1;
            const C zm   = r[p + m * TD];
            const C zc   = r[p + (LD - m) * TD];
            C x;
            if ((row & 1) == 0)
                x = C{(R)0.5 * (zm.x + zc.x), (R)0.5 * (zm.y - zc.y)};   // (Z_m + conj(Z_{L-m}))/2
            else
                x = C{(R)0.5 * (zm.y + zc.y), (R)0.5 * (zc.x - zm.x)};   // (Z_m - conj(Z_{L-m}))/(2i)
            const int i = rr / ny, j = rr - i * ny;
            S_out[((size_t)i * 2 * ny + j) * NZ + (m - 1)] = x;
        }
    }

    // ---- norm of psi' (imaginary time): deterministic two-level reduction ---
    if (MODE == ZM_IT_MID) {
        for (int off = 16; off > 0; off >>= 1)
            acc += __shfl_down_sync(0xffffffffu, acc, off);
        if ((tid & 31) == 0)
            red[tid >> 5] = acc;
        __syncthreads();
        __shared__ bool last;
        if (tid == 0) {
            double v = 0;
            for (int w = 0; w < NT / 32; ++w)
                v += red[w];
            a.partial[blockIdx.x] = v;
            __threadfence();
            const unsigned t = atomicAdd(a.ticket, 1u);
            last             = (t == gridDim.x - 1);
        }
        __syncthreads();
        if (last) {
            __threadfence();
            double v = 0;
            for (int b = tid; b < (int)gridDim.x; b += NT)
                v += ((volatile double *)a.partial)[b];
            for (int off = 16; off > 0; off >>= 1)
                v += __shfl_down_sync(0xffffffffu, v, off);
            if ((tid & 31) == 0)
                red[tid >> 5] = v;
            __syncthreads();
            if (tid == 0) {
                double x = 0;
                for (int w = 0; w < NT / 32; ++w)
                    x += red[w];
                x *= a.dV;
                a.norm_state[0] = x;
                a.norm_state[1] = x;
                if (!(x > 0.0) || !isfinite(x))
                    a.status[0] = 1;
                *a.ticket = 0u;
            }
        }
    }
}

// Shared memory of k2_z<R, NZ, *>.
template <class R, int NZ> constexpr size_t z_smem() {
    return sizeof(cplx<R>) * (33 * NZ + 17 * 2 * NZ) + sizeof(R) * 2 * 33 * NZ;
}

} // namespace gpe
