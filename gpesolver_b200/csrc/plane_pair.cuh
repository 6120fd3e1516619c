// The plane kernels on a cluster of two CTAs per x plane.
//
// k4_yz (fused_yz.cuh) runs one CTA per x plane: 128 planes at 128 x 128 x 32
// leave 20 of the 148 SMs idle, and its 152 KB of shared memory keep one CTA
// (one barrier domain) per SM, so the shared-memory phases of the transforms
// and their arithmetic cannot overlap.  k5_yz_pair splits each plane between
// the two CTAs of a cluster, each with half the shared memory (two CTAs per SM,
// 2 nx CTAs in all):
//
//   A  CTA r holds the kz columns [r nz/2, (r+1) nz/2) of the dipolar spectrum
//      (2ny rows) and of the kinetic increment (ny rows) and runs the inverse y
//      transforms on them; the last stage of each sends the rows of the other
//      CTA's half straight into that CTA's shared memory (distributed shared
//      memory, stores through map_shared_rank) and keeps its own;
//   (cluster barrier)
//   C  CTA r holds the rows [r ny/2, (r+1) ny/2) of both planes: dipolar C2R_z
//      (row pairs) -> V + cdd phi, kinetic iFFT_z, + kept psi, the merged phase
//      step, rho, FFT_z and R2C_z; the last stages again send the other CTA's
//      columns to it;
//   (cluster barrier)
//   E  forward y transforms on the column halves, stored to global memory.
//
// The arithmetic of every line is that of k4_yz (same radices, twiddles and
// order of operations).  Only the middle iterations of a call run here
// (ZM_RT_MID, ZM_IT_MID); the first and the last stay on k4_yz.
//
// Shared memory of one CTA of k5_yz_pair (complex C = 8 bytes in FP32; strides
// odd):
//   XD  2ny rows x (nz/2 + 1): dipolar column half (A), then the forward
//       dipolar tile (E, rows < ny written in C); during C its upper half holds
//       DP, the row-pair lines of the real transforms (nothing is sent there)
//   XK   ny rows x (nz/2 + 1): kinetic column half (A), forward tile (E)
//   ZD   ny/2 rows x (nz + 1): dipolar row half (filled in A by both CTAs)
//   ZK   ny/2 rows x (nz + 1): kinetic row half (filled in A by both CTAs)
//   RP   ny/2 rows x (nz + 1): kept real-space psi of this CTA's rows
//   FP   V + cdd phi, then rho, of this CTA's rows (even rows, then odd rows)
// The partner writes only ZD, ZK (before the first cluster barrier; nothing
// here reads them before it) and the lower half of XD and XK (after the first
// barrier, by which this CTA has finished reading them; until the second
// barrier this CTA itself uses only the upper half of XD there).
#pragma once

#include <cooperative_groups.h>

#include "fused_yz.cuh"

namespace gpe {

template <class R, int NY, int NZ> struct PairShape {
    using C                    = cplx<R>;
    static constexpr int NZH   = NZ / 2;  // kz columns per CTA (y transforms)
    static constexpr int NYH   = NY / 2;  // rows per CTA (z transforms)
    static constexpr int PC    = NZH + 1; // row stride of the column tiles XD, XK
    static constexpr int PZ    = NZ + 1;  // row stride of the row tiles ZD, ZK, RP
    static constexpr int NPP   = NYH / 2; // row pairs of the real z transforms
    static constexpr int LD    = 2 * NZ;  // real-transform line length
    static constexpr int TD    = NPP + 1; // DP element stride
    static constexpr int FS    = NZ + 1;  // FP row stride (floats)
    // odd rows 16 banks after the even rows (as in YZShape)
    static constexpr int FH    = NPP * FS + (((16 - (NPP * FS) % 32) % 32) + 32) % 32;
    static constexpr int FPN   = FH + NPP * FS;
    static constexpr size_t XD_B   = sizeof(C) * 2 * NY * PC;
    static constexpr size_t XK_B   = sizeof(C) * NY * PC;
    static constexpr size_t Z_B    = sizeof(C) * NYH * PZ;
    static constexpr size_t OFF_XK = XD_B;
    static constexpr size_t OFF_ZD = OFF_XK + XK_B;
    static constexpr size_t OFF_ZK = OFF_ZD + Z_B;
    static constexpr size_t OFF_RP = OFF_ZK + Z_B;
    static constexpr size_t OFF_FP = OFF_RP + Z_B;
    static constexpr size_t OFF_DP = sizeof(C) * NY * PC; // upper half of XD
    static constexpr size_t SMEM   = OFF_FP + sizeof(R) * FPN;
    static_assert(NZ % 4 == 0 && NY % 4 == 0, "halves of even row pairs and columns");
    static_assert(sizeof(C) * TD * LD <= XD_B - OFF_DP, "DP fits in the upper half of XD");
    // half the one-CTA kernel's threads, at least 128, whole warps (the norm
    // reduction of k5_yz_pair_it shuffles over full warps)
    static constexpr int NT0 = YZShape<R, NY, NZ>::NT / 2;
    static constexpr int NT  = NT0 < 128 ? 128 : (NT0 + 31) / 32 * 32;
    static_assert(NT % 32 == 0, "whole warps");
    static __device__ __forceinline__ int fpi(int r, int k) { return (r & 1) * FH + (r >> 1) * FS + k; }
};

// C2R row-pair lines of the row half in ZD -> DP: z[m] = X_a[m] + i X_b[m] over
// the full 2nz-point spectrum (bins 1..nz stored at kz - 1, bin 0 zero, bins > nz
// by symmetry)
template <class R, int NY, int NZ, int NT>
__device__ __forceinline__ void pair_lines_c2r(cplx<R> *DP, const cplx<R> *ZD, int tid) {
    using C  = cplx<R>;
    using G  = PairShape<R, NY, NZ>;
    constexpr int NPP = G::NPP, LD = G::LD, TD = G::TD, PZ = G::PZ;
    for (int e = tid; e < NPP * LD; e += NT) {
        const int m = e % LD, p = e / LD;
        C z         = C{(R)0, (R)0};
        if (m > 0) {
            const int mm = m <= NZ ? m : LD - m;
            const C xa   = ZD[(2 * p) * PZ + mm - 1];
            const C xb   = ZD[(2 * p + 1) * PZ + mm - 1];
            if (m == NZ)
                z = C{xa.x, xb.x}; // self-conjugate bin: real parts only
            else if (m < NZ)
                z = C{xa.x - xb.y, xa.y + xb.x};
            else
                z = C{xa.x + xb.y, xb.x - xa.y};
        }
        DP[p + m * TD] = z;
    }
}

// R2C unpacking of the row half's pair lines in DP: bin m (1..nz) of local row
// y goes to the CTA that owns column m - 1 (XD local, XDo the partner's).
template <class R, int NY, int NZ, int NT>
__device__ __forceinline__ void pair_unpack_r2c(cplx<R> *XD, cplx<R> *XDo, const cplx<R> *DP, int r, int tid) {
    using C  = cplx<R>;
    using G  = PairShape<R, NY, NZ>;
    constexpr int NYH = G::NYH, NZH = G::NZH, LD = G::LD, TD = G::TD, PC = G::PC;
    const int y0 = r * NYH;
    for (int e = tid; e < NYH * NZ; e += NT) {
        const int y = e / NZ, m = e - y * NZ + 1;
        const int p = y >> 1;
        const C zm  = DP[p + m * TD];
        const C zc  = DP[p + (LD - m) * TD];
        C x;
        if ((y & 1) == 0)
            x = C{(R)0.5 * (zm.x + zc.x), (R)0.5 * (zm.y - zc.y)}; // (Z_m + conj(Z_{L-m}))/2
        else
            x = C{(R)0.5 * (zm.y + zc.y), (R)0.5 * (zc.x - zm.x)}; // (Z_m - conj(Z_{L-m}))/(2i)
        C *d = ((m - 1 >= NZH) == (r == 1)) ? XD : XDo;
        d[(y0 + y) * PC + ((m - 1) % NZH)] = x;
    }
}

template <class R, int NY, int NZ>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(PairShape<R, NY, NZ>::NT, 2)
    k5_yz_pair(ZArgs a, YZTwid tw) {
    namespace cg   = cooperative_groups;
    using C        = cplx<R>;
    using G        = PairShape<R, NY, NZ>;
    constexpr int NT = G::NT, NZH = G::NZH, NYH = G::NYH, PC = G::PC, PZ = G::PZ;
    constexpr int NPP = G::NPP, LD = G::LD, TD = G::TD;
    cg::cluster_group cl = cg::this_cluster();
    const int r          = (int)cl.block_rank(); // 0 or 1
    const int tid        = threadIdx.x;
    const int i          = blockIdx.x >> 1; // x plane
    const int nx         = a.nx;
    const int c0         = r * NZH; // first kz column of this CTA
    const int y0         = r * NYH; // first row of this CTA

    C *XD = reinterpret_cast<C *>(g_smem);
    C *XK = reinterpret_cast<C *>(g_smem + G::OFF_XK);
    C *ZD = reinterpret_cast<C *>(g_smem + G::OFF_ZD);
    C *ZK = reinterpret_cast<C *>(g_smem + G::OFF_ZK);
    C *RP = reinterpret_cast<C *>(g_smem + G::OFF_RP);
    R *FP = reinterpret_cast<R *>(g_smem + G::OFF_FP);
    C *DP = reinterpret_cast<C *>(g_smem + G::OFF_DP);
    // the partner's tiles (distributed shared memory)
    C *XDo = cl.map_shared_rank(XD, r ^ 1);
    C *XKo = cl.map_shared_rank(XK, r ^ 1);
    C *ZDo = cl.map_shared_rank(ZD, r ^ 1);
    C *ZKo = cl.map_shared_rank(ZK, r ^ 1);

    const size_t pl = (size_t)i * NY * NZ;
    const C *Q_g    = reinterpret_cast<const C *>(a.psi_in) + pl; // kinetic increment (ky, kz)
    C *P_o          = reinterpret_cast<C *>(a.psi_out) + pl;      // psi spectrum out (ky, kz)
    C *Pr_g         = reinterpret_cast<C *>(a.psi_r) + pl + (size_t)y0 * NZ;
    const R *V_g    = reinterpret_cast<const R *>(a.V) + pl + (size_t)y0 * NZ;
    C *S_g          = reinterpret_cast<C *>(a.S) + (size_t)i * 2 * NY * NZ;
    const R cdd     = (R)a.cdd;
    const C *dyt = (const C *)tw.dy.tw, *dyl = (const C *)tw.dy.lo;
    const C *dzt = (const C *)tw.dz.tw, *dzl = (const C *)tw.dz.lo;
    const C *kyt = (const C *)tw.ky.tw, *kyl = (const C *)tw.ky.lo;
    const C *kzt = (const C *)tw.kz.tw, *kzl = (const C *)tw.kz.lo;
    // the step coefficients of this and the next iteration, read first (two
    // dependent L2 reads that land behind the plane loads)
    R g3, gw;
    {
        const int base     = *a.step.base + a.step.local;
        const StepCoef c0c = a.step.coef[base];
        const StepCoef c1c = a.step.coef[base + 1];
        g3                 = (R)(c0c.g3w + c1c.g3w);
        gw                 = (R)(c0c.gw15 + c1c.gw15);
    }

    // ---- loads: the column halves of both spectra; V and the kept psi of this
    // CTA's rows (needed from the C2R's last stage on) ----------------------
#pragma unroll 4
    for (int e = tid; e < 2 * NY * NZH; e += NT) {
        const int row = e / NZH, c = e - row * NZH;
        cp_async8(&XD[row * PC + c], &S_g[row * NZ + c0 + c]);
    }
#pragma unroll 4
    for (int e = tid; e < NY * NZH; e += NT) {
        const int row = e / NZH, c = e - row * NZH;
        cp_async8(&XK[row * PC + c], &Q_g[row * NZ + c0 + c]);
    }
    cp_async_commit();
#pragma unroll 4
    for (int e = tid; e < NYH * NZ; e += NT) {
        const int row = e / NZ, k = e - row * NZ;
        cp_async4(&FP[G::fpi(row, k)], &V_g[e]);
        cp_async8(&RP[row * PZ + k], &Pr_g[e]);
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();

    // ---- A: inverse y transforms of the column halves ------------------------
    {
        using DYI = PlanePass<+1, R, 2 * NY, NZH, 1, PC, NT, false, true, false, true>;
        using KYI = PlanePass<+1, R, NY, NZH, 1, PC, NT, true, false>;
        joint_stages<DYI, 0, DYI::NSTG - 1, KYI, 0, KYI::NSTG - 1>(XD, dyt, dyl, XK, kyt, kyl, tid);
        typename DYI::Last::Regs da;
        typename KYI::Last::Regs ka;
        DYI::Last::read(XD, da, dyt, dyl, tid);
        KYI::Last::read(XK, ka, kyt, kyl, tid);
        // row y of column c goes to the CTA that owns row y
#pragma unroll
        for (int rd = 0; rd < DYI::Last::ROUNDS; ++rd) {
            if (!DYI::Last::valid(rd * NT + tid))
                break;
            const int c = c0 + DYI::Last::line(tid, rd);
#pragma unroll
            for (int q = 0; q < DYI::Last::RADIX; ++q) {
                if (2 * q >= DYI::Last::RADIX) // pruned: only rows < ny are kept
                    continue;
                const int y = DYI::Last::elem(tid, rd, q);
                C *d        = ((y >= NYH) == (r == 1)) ? ZD : ZDo;
                d[(y % NYH) * PZ + c] = da[rd][q];
            }
        }
#pragma unroll
        for (int rd = 0; rd < KYI::Last::ROUNDS; ++rd) {
            if (!KYI::Last::valid(rd * NT + tid))
                break;
            const int c = c0 + KYI::Last::line(tid, rd);
#pragma unroll
            for (int q = 0; q < KYI::Last::RADIX; ++q) {
                const int y = KYI::Last::elem(tid, rd, q);
                C *d        = ((y >= NYH) == (r == 1)) ? ZK : ZKo;
                d[(y % NYH) * PZ + c] = ka[rd][q];
            }
        }
    }
    cp_async_wait<0>(); // V and the kept psi: visible to the block after the barriers below
    cl.sync();          // ZD, ZK complete in both CTAs

    // ---- C: z work on the row halves -------------------------------------------
    using C2R = PlanePass<+1, R, LD, NPP, 1, TD, NT, false, true, false, true>;
    using ZI  = PlanePass<+1, R, NZ, NYH, PZ, 1, NT, true, false>;
    using ZF  = PlanePass<-1, R, NZ, NYH, PZ, 1, NT, true, true>;
    using R2C = PlanePass<-1, R, LD, NPP, 1, TD, NT, false, false, true, false>;
    static_assert(ZI::Last::RADIX == ZF::First::RADIX && ZI::Last::ROUNDS == ZF::First::ROUNDS &&
                      ZI::Last::ITEMS == ZF::First::ITEMS,
                  "paired z transforms share the register layout");
    pair_lines_c2r<R, NY, NZ, NT>(DP, ZD, tid);
    __syncthreads();
    // C2R || kinetic iFFT_z, all stages but the last
    joint_stages<C2R, 0, C2R::NSTG - 1, ZI, 0, ZI::NSTG - 1>(DP, dzt, dzl, ZK, kzt, kzl, tid);
    typename ZI::Last::Regs zr;
    {
        // last C2R stage -> FP = V + cdd phi; last iFFT_z stage -> registers
        typename C2R::Last::Regs ca;
        C2R::Last::read(DP, ca, dzt, dzl, tid);
        ZI::Last::read(ZK, zr, kzt, kzl, tid);
#pragma unroll
        for (int rd = 0; rd < C2R::Last::ROUNDS; ++rd) {
            if (!C2R::Last::valid(rd * NT + tid))
                break;
            const int p = C2R::Last::line(tid, rd);
#pragma unroll
            for (int q = 0; q < C2R::Last::RADIX; ++q) {
                if (2 * q >= C2R::Last::RADIX) // pruned: z >= nz is not kept
                    continue;
                const int k = C2R::Last::elem(tid, rd, q);
                const C v   = ca[rd][q];
                FP[G::fpi(2 * p, k)] += cdd * v.x;
                FP[G::fpi(2 * p + 1, k)] += cdd * v.y;
            }
        }
    }
    __syncthreads(); // FP = V + cdd phi

    // merged potential half steps of two consecutive iterations:
    // theta = -dt/2 [2 (V + cdd phi) + g3 |psi|^2 + gw |psi|^3]
    const R cV = (R)2, hdt = (R)a.half_dt, wat = (R)a.w_atoms;
    const bool xin = i >= 1 && i < nx - 1;
#pragma unroll
    for (int rd = 0; rd < ZI::Last::ROUNDS; ++rd) {
        if (!ZI::Last::valid(rd * NT + tid))
            break;
        const int y  = ZI::Last::line(tid, rd); // row within this CTA's half
        const int yg = y0 + y;
#pragma unroll
        for (int q = 0; q < ZI::Last::RADIX; ++q) {
            const int z = ZI::Last::elem(tid, rd, q);
            const int f = G::fpi(y, z);
            // psi = kept psi + kinetic increment, then the phase step
            C p = cadd(zr[rd][q], RP[y * PZ + z]);
            if (xin && yg >= 1 && yg < NY - 1 && z >= 1 && z < NZ - 1) {
                const R dens  = p.x * p.x + p.y * p.y;
                const R am    = sqrt(dens);
                const R total = cV * FP[f] + g3 * dens + gw * (am * am * am);
                R s, c;
                sincos_r<R>((R)-0.5 * hdt * total, &s, &c);
                p = apply_wm1(p, C{(R)-2 * s * s, (R)2 * s * c});
            }
            FP[f]          = wat * (p.x * p.x + p.y * p.y); // rho for the next dipolar spectrum
            RP[y * PZ + z] = p;
            zr[rd][q]      = p;
        }
    }
    __syncthreads(); // rho and the new psi complete

    // R2C pair lines from rho (upper half zero); first FFT_z stage from the
    // registers (the iFFT_z reads of ZK are behind the barriers above)
    for (int e = tid; e < NPP * NZ; e += NT) {
        const int m = e % NZ, p = e / NZ;
        DP[p + m * TD] = C{FP[G::fpi(2 * p, m)], FP[G::fpi(2 * p + 1, m)]};
    }
#pragma unroll
    for (int rd = 0; rd < ZF::First::ROUNDS; ++rd) {
        if (!ZF::First::valid(rd * NT + tid))
            break;
        DFT<ZF::First::RADIX, -1, R, true>::run(zr[rd]);
    }
    // bin kz of row y of the finished FFT_z goes to the CTA owning column kz
    // (XK's lower part: nothing reads it between the two cluster barriers)
    auto emit_kz = [&](const auto &v, int rd, int line, auto elem) {
        const int yg = y0 + line;
#pragma unroll
        for (int q = 0; q < (int)(sizeof(v[0]) / sizeof(v[0][0])); ++q) {
            const int kz = elem(q);
            C *d         = ((kz >= NZH) == (r == 1)) ? XK : XKo;
            d[yg * PC + (kz % NZH)] = v[rd][q];
        }
    };
    if constexpr (ZF::NSTG == 1) {
        // a single-stage z transform (nz = 16) is finished in the registers
#pragma unroll
        for (int rd = 0; rd < ZF::First::ROUNDS; ++rd) {
            if (!ZF::First::valid(rd * NT + tid))
                break;
            emit_kz(zr, rd, ZF::First::line(tid, rd), [&](int q) { return ZF::First::elem(tid, rd, q); });
        }
        __syncthreads(); // DP (R2C pair lines) complete
        plane_out<R, NYH, NZ, PZ, NT>(Pr_g, RP, tid); // kept psi for the next iteration
        R2C::template stages<0, R2C::NSTG>(DP, dzt, dzl, tid);
        pair_unpack_r2c<R, NY, NZ, NT>(XD, XDo, DP, r, tid);
    } else {
        ZF::First::write(ZK, zr, tid);
        __syncthreads();
        plane_out<R, NYH, NZ, PZ, NT>(Pr_g, RP, tid); // kept psi for the next iteration
        joint_stages<R2C, 0, R2C::NSTG, ZF, 1, ZF::NSTG - 1>(DP, dzt, dzl, ZK, kzt, kzl, tid);
        // last FFT_z stage, emitted to the column owners
        typename ZF::Last::Regs fa;
        ZF::Last::read(ZK, fa, kzt, kzl, tid);
#pragma unroll
        for (int rd = 0; rd < ZF::Last::ROUNDS; ++rd) {
            if (!ZF::Last::valid(rd * NT + tid))
                break;
            emit_kz(fa, rd, ZF::Last::line(tid, rd), [&](int q) { return ZF::Last::elem(tid, rd, q); });
        }
        pair_unpack_r2c<R, NY, NZ, NT>(XD, XDo, DP, r, tid);
    }
    cl.sync(); // forward tiles complete in both CTAs

    // ---- E: forward y transforms of the column halves -> global ---------------
    {
        using DYF = PlanePass<-1, R, 2 * NY, NZH, 1, PC, NT, false, false, true, false>;
        using KYF = PlanePass<-1, R, NY, NZH, 1, PC, NT, true, false>;
        joint_stages<DYF, 0, DYF::NSTG - 1, KYF, 0, KYF::NSTG - 1>(XD, dyt, dyl, XK, kyt, kyl, tid);
        typename DYF::Last::Regs da;
        DYF::Last::read(XD, da, dyt, dyl, tid);
#pragma unroll
        for (int rd = 0; rd < DYF::Last::ROUNDS; ++rd) {
            if (!DYF::Last::valid(rd * NT + tid))
                break;
            const int c = c0 + DYF::Last::line(tid, rd);
#pragma unroll
            for (int q = 0; q < DYF::Last::RADIX; ++q)
                S_g[DYF::Last::elem(tid, rd, q) * NZ + c] = da[rd][q];
        }
        typename KYF::Last::Regs kb;
        KYF::Last::read(XK, kb, kyt, kyl, tid);
#pragma unroll
        for (int rd = 0; rd < KYF::Last::ROUNDS; ++rd) {
            if (!KYF::Last::valid(rd * NT + tid))
                break;
            const int c = c0 + KYF::Last::line(tid, rd);
#pragma unroll
            for (int q = 0; q < KYF::Last::RADIX; ++q)
                P_o[KYF::Last::elem(tid, rd, q) * NZ + c] = kb[rd][q];
        }
    }
}

// Imaginary time (the middle iterations of imag_steps, ZM_IT_MID) on the same
// two-CTA split: A inverse y transform of the dipolar column half, rows sent to
// their owner; C the C2R of the row pairs -> phi, the Euler stencil step of this
// CTA's rows (psi rows y0 - 1 .. y0 + ny/2 of this plane and the same rows of
// the two x neighbours, copied in from global memory), rho, R2C, columns sent to
// their owner; E forward y transform -> spectrum.  The norm of psi' is reduced
// over all 2 nx CTAs (partial sums; the last CTA to finish sums them in a fixed
// order).
//
// Shared memory of one CTA:
//   XD  2ny rows x (nz/2 + 1): dipolar column half, then the forward tile; DP
//       (row-pair lines) in its upper half during C
//   ZD  ny/2 rows x (nz + 1): dipolar row half (filled in A by both CTAs)
//   PH  ny/2 + 2 rows x (nz + 1): psi rows y0 - 1 .. y0 + ny/2 of this plane
//   XM, XP  ny/2 rows x (nz + 1): psi rows y0 .. y0 + ny/2 - 1 of planes i -+ 1
//   FP  V + cdd phi, then rho, of this CTA's rows
template <class R, int NY, int NZ> struct PairShapeIT {
    using G                        = PairShape<R, NY, NZ>;
    using C                        = cplx<R>;
    static constexpr size_t PH_B   = sizeof(C) * (G::NYH + 2) * G::PZ;
    static constexpr size_t OFF_ZD = G::XD_B;
    static constexpr size_t OFF_PH = OFF_ZD + G::Z_B;
    static constexpr size_t OFF_XM = OFF_PH + PH_B;
    static constexpr size_t OFF_XP = OFF_XM + G::Z_B;
    static constexpr size_t OFF_FP = OFF_XP + G::Z_B;
    static constexpr size_t SMEM   = OFF_FP + sizeof(R) * G::FPN;
};

template <class R, int NY, int NZ>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(PairShape<R, NY, NZ>::NT, 2)
    k5_yz_pair_it(ZArgs a, YZTwid tw) {
    namespace cg   = cooperative_groups;
    using C        = cplx<R>;
    using G        = PairShape<R, NY, NZ>;
    using GI       = PairShapeIT<R, NY, NZ>;
    constexpr int NT = G::NT, NZH = G::NZH, NYH = G::NYH, PC = G::PC, PZ = G::PZ;
    constexpr int NPP = G::NPP, LD = G::LD, TD = G::TD;
    cg::cluster_group cl = cg::this_cluster();
    const int r          = (int)cl.block_rank();
    const int tid        = threadIdx.x;
    const int i          = blockIdx.x >> 1; // x plane
    const int nx         = a.nx;
    const int c0         = r * NZH;
    const int y0         = r * NYH;
    __shared__ double red[NT / 32];
    __shared__ bool last;

    C *XD  = reinterpret_cast<C *>(g_smem);
    C *ZD  = reinterpret_cast<C *>(g_smem + GI::OFF_ZD);
    C *PH  = reinterpret_cast<C *>(g_smem + GI::OFF_PH);
    C *XM  = reinterpret_cast<C *>(g_smem + GI::OFF_XM);
    C *XP  = reinterpret_cast<C *>(g_smem + GI::OFF_XP);
    R *FP  = reinterpret_cast<R *>(g_smem + GI::OFF_FP);
    C *DP  = reinterpret_cast<C *>(g_smem + G::OFF_DP);
    C *XDo = cl.map_shared_rank(XD, r ^ 1);
    C *ZDo = cl.map_shared_rank(ZD, r ^ 1);

    const size_t pln = (size_t)NY * NZ;
    const size_t pl  = (size_t)i * pln;
    const C *pin     = reinterpret_cast<const C *>(a.psi_in);
    C *pout          = reinterpret_cast<C *>(a.psi_out);
    const C *bnd     = reinterpret_cast<const C *>(a.bnd);
    const R *V_g     = reinterpret_cast<const R *>(a.V) + pl + (size_t)y0 * NZ;
    R *phi_g         = reinterpret_cast<R *>(a.phi) + pl + (size_t)y0 * NZ;
    C *S_g           = reinterpret_cast<C *>(a.S) + (size_t)i * 2 * NY * NZ;
    const R cdd      = (R)a.cdd;
    const bool xin   = i >= 1 && i < nx - 1;
    const C *dyt = (const C *)tw.dy.tw, *dyl = (const C *)tw.dy.lo;
    const C *dzt = (const C *)tw.dz.tw, *dzl = (const C *)tw.dz.lo;
    // the stencil's step coefficients and the kept boundary values of this
    // thread's stencil points, read first (behind the plane loads; every row
    // has its two z-boundary points)
    const StepCoef cf = a.step.coef[0];
    constexpr int SE  = (NYH * NZ + NT - 1) / NT; // stencil points per thread
    C bpre[SE];
#pragma unroll
    for (int j = 0; j < SE; ++j) {
        const int e = tid + j * NT;
        const int rl = e / NZ, k = e - rl * NZ, y = y0 + rl;
        if (e < NYH * NZ && (!xin || y < 1 || y >= NY - 1 || k < 1 || k >= NZ - 1))
            bpre[j] = __ldg(&bnd[pl + (size_t)y * NZ + k]);
    }

    // ---- loads: the dipolar column half; V, the psi rows of the stencil ------
#pragma unroll 4
    for (int e = tid; e < 2 * NY * NZH; e += NT) {
        const int row = e / NZH, c = e - row * NZH;
        cp_async8(&XD[row * PC + c], &S_g[row * NZ + c0 + c]);
    }
    cp_async_commit();
#pragma unroll 4
    for (int e = tid; e < NYH * NZ; e += NT) {
        const int row = e / NZ, k = e - row * NZ;
        cp_async4(&FP[G::fpi(row, k)], &V_g[e]);
    }
    {
        // rows y0 - 1 .. y0 + ny/2 of this plane, those inside the grid (PH row
        // 0 is row y0 - 1)
        const int ylo = y0 > 0 ? y0 - 1 : 0, yhi = y0 + NYH < NY ? y0 + NYH : NY - 1;
        const C *src  = pin + pl + (size_t)ylo * NZ;
        for (int e = tid; e < (yhi - ylo + 1) * NZ; e += NT) {
            const int row = e / NZ, k = e - row * NZ;
            cp_async8(&PH[(ylo + row - (y0 - 1)) * PZ + k], &src[e]);
        }
    }
    if (xin) {
        const C *sm = pin + pl - pln + (size_t)y0 * NZ, *sp = pin + pl + pln + (size_t)y0 * NZ;
#pragma unroll 4
        for (int e = tid; e < NYH * NZ; e += NT) {
            const int row = e / NZ, k = e - row * NZ;
            cp_async8(&XM[row * PZ + k], &sm[e]);
            cp_async8(&XP[row * PZ + k], &sp[e]);
        }
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();

    // ---- A: inverse y transform of the dipolar column half ---------------------
    {
        using DYI = PlanePass<+1, R, 2 * NY, NZH, 1, PC, NT, false, true, false, true>;
        DYI::template stages<0, DYI::NSTG - 1>(XD, dyt, dyl, tid);
        typename DYI::Last::Regs da;
        DYI::Last::read(XD, da, dyt, dyl, tid);
#pragma unroll
        for (int rd = 0; rd < DYI::Last::ROUNDS; ++rd) {
            if (!DYI::Last::valid(rd * NT + tid))
                break;
            const int c = c0 + DYI::Last::line(tid, rd);
#pragma unroll
            for (int q = 0; q < DYI::Last::RADIX; ++q) {
                if (2 * q >= DYI::Last::RADIX) // pruned: only rows < ny are kept
                    continue;
                const int y = DYI::Last::elem(tid, rd, q);
                C *d        = ((y >= NYH) == (r == 1)) ? ZD : ZDo;
                d[(y % NYH) * PZ + c] = da[rd][q];
            }
        }
    }
    cp_async_wait<0>();
    cl.sync(); // ZD complete in both CTAs

    // ---- C: phi, the stencil step and rho of this CTA's rows -------------------
    using C2R = PlanePass<+1, R, LD, NPP, 1, TD, NT, false, true, false, true>;
    using R2C = PlanePass<-1, R, LD, NPP, 1, TD, NT, false, false, true, false>;
    pair_lines_c2r<R, NY, NZ, NT>(DP, ZD, tid);
    __syncthreads();
    C2R::template stages<0, C2R::NSTG - 1>(DP, dzt, dzl, tid);
    {
        typename C2R::Last::Regs ca;
        C2R::Last::read(DP, ca, dzt, dzl, tid);
#pragma unroll
        for (int rd = 0; rd < C2R::Last::ROUNDS; ++rd) {
            if (!C2R::Last::valid(rd * NT + tid))
                break;
            const int p = C2R::Last::line(tid, rd);
#pragma unroll
            for (int q = 0; q < C2R::Last::RADIX; ++q) {
                if (2 * q >= C2R::Last::RADIX) // pruned: z >= nz is not kept
                    continue;
                const int k = C2R::Last::elem(tid, rd, q);
                const C v   = ca[rd][q];
                phi_g[(2 * p) * NZ + k]     = v.x;
                phi_g[(2 * p + 1) * NZ + k] = v.y;
                FP[G::fpi(2 * p, k)] += cdd * v.x;
                FP[G::fpi(2 * p + 1, k)] += cdd * v.y;
            }
        }
    }
    __syncthreads(); // FP = V + cdd phi

    double acc = 0.0;
    {
        // psi_in / sqrt(divisor): the Euler step of imag_iter_linear_step +
        // imag_iter_nonlinear_step on the interior, the kept boundary values
        // elsewhere
        const R sc        = (R)(1.0 / sqrt(a.norm_state[1]));
        const R wat       = (R)a.w_atoms;
        const R g3w = (R)cf.g3w, gw15 = (R)cf.gw15;
        const R cx = (R)a.cx, cy = (R)a.cy, cz = (R)a.cz, dtau = (R)a.dtau;
#pragma unroll
        for (int j = 0; j < SE; ++j) {
            const int e = tid + j * NT;
            if (SE * NT != NYH * NZ && e >= NYH * NZ)
                break;
            const int rl   = e / NZ, k = e - rl * NZ;
            const int y    = y0 + rl;
            const size_t q = pl + (size_t)y * NZ + k;
            C o;
            if (!xin || y < 1 || y >= NY - 1 || k < 1 || k >= NZ - 1) {
                o = bpre[j]; // bnd[q], read at kernel start
            } else {
                const C *pp = PH + (rl + 1) * PZ + k;
                const C c0v = cscale(pp[0], sc);
                const C xm = cscale(XM[rl * PZ + k], sc), xp = cscale(XP[rl * PZ + k], sc);
                const C ym = cscale(pp[-PZ], sc), yp = cscale(pp[PZ], sc);
                const C zm = cscale(pp[-1], sc), zp = cscale(pp[1], sc);
                const R vv   = FP[G::fpi(rl, k)];
                const R dens = c0v.x * c0v.x + c0v.y * c0v.y;
                const R am   = sqrt(dens);
                const R nl   = g3w * dens + gw15 * (am * am * am);
                const R lr   = cx * ((xm.x + xp.x) - 2 * c0v.x) - cy * ((ym.x + yp.x) - 2 * c0v.x) -
                             cz * ((zm.x + zp.x) - 2 * c0v.x) + c0v.x * vv + nl * c0v.x;
                const R li = cx * ((xm.y + xp.y) - 2 * c0v.y) - cy * ((ym.y + yp.y) - 2 * c0v.y) -
                             cz * ((zm.y + zp.y) - 2 * c0v.y) + c0v.y * vv + nl * c0v.y;
                o = C{c0v.x - dtau * lr, c0v.y - dtau * li};
            }
            pout[q] = o;
            acc += (double)o.x * o.x + (double)o.y * o.y;
            FP[G::fpi(rl, k)] = wat * (o.x * o.x + o.y * o.y);
        }
    }
    __syncthreads(); // rho complete

    // R2C of rho (row pairs), bins sent to the CTA owning their column
    for (int e = tid; e < NPP * NZ; e += NT) {
        const int m = e % NZ, p = e / NZ;
        DP[p + m * TD] = C{FP[G::fpi(2 * p, m)], FP[G::fpi(2 * p + 1, m)]};
    }
    __syncthreads();
    R2C::template stages<0, R2C::NSTG>(DP, dzt, dzl, tid);
    pair_unpack_r2c<R, NY, NZ, NT>(XD, XDo, DP, r, tid);
    cl.sync(); // forward tiles complete in both CTAs

    // ---- E: forward y transform of the dipolar column half -> spectrum --------
    {
        using DYF = PlanePass<-1, R, 2 * NY, NZH, 1, PC, NT, false, false, true, false>;
        DYF::template stages<0, DYF::NSTG - 1>(XD, dyt, dyl, tid);
        typename DYF::Last::Regs da;
        DYF::Last::read(XD, da, dyt, dyl, tid);
#pragma unroll
        for (int rd = 0; rd < DYF::Last::ROUNDS; ++rd) {
            if (!DYF::Last::valid(rd * NT + tid))
                break;
            const int c = c0 + DYF::Last::line(tid, rd);
#pragma unroll
            for (int q = 0; q < DYF::Last::RADIX; ++q)
                S_g[DYF::Last::elem(tid, rd, q) * NZ + c] = da[rd][q];
        }
    }

    // ---- norm of psi': deterministic two-level reduction over the 2 nx CTAs ---
    for (int off = 16; off > 0; off >>= 1)
        acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((tid & 31) == 0)
        red[tid >> 5] = acc;
    __syncthreads();
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

} // namespace gpe
