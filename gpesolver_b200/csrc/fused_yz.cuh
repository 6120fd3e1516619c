// One kernel per x plane for everything between two x passes.
//
// After the x pass, each x plane of psi (ny x nz, ky kz spectrum) and of the
// dipolar spectrum (2ny x nz) is independent of the others until the next x
// pass.  k4_yz keeps one plane of each in shared memory and runs, for plane i,
//
//   dipolar  iFFT_y(2ny, lower half kept) -> C2R_z (row pairs) -> phi
//   kinetic  iFFT_y(ny) -> iFFT_z(nz) -> + psi_r -> phase -> FFT_z(nz) -> FFT_y(ny)
//   dipolar  rho -> R2C_z (row pairs) -> FFT_y(2ny, upper half zero)
//
// (imaginary time: the Euler stencil step in place of the kinetic transforms).
// In real time the x pass hands over the kinetic increment (fused.cuh,
// k3_x_kin): its inverse yz transform is added to the real-space psi that the
// previous plane kernel kept (psi_r, its own copy of the plane after the
// phase step), and the new psi after the phase goes back to psi_r,
// so one iteration is two kernels (x pass, yz plane) instead of four; the three
// plane passes no longer go through global memory between each other.  The
// z-line transforms pair through registers (iFFT_z ends, the phase is applied,
// FFT_z starts, without a shared-memory round trip).
//
// Shared memory (complex C = 8 bytes in FP32), row stride PS = nz + 1 (odd:
// conflict-free for both the y columns and the z rows):
//   SP  2ny rows x PS  dipolar plane (ky or y, kz - 1)
//   PP   ny rows x PS  psi plane (ky or y, kz or z)            (real time)
//   FP   ny rows x (nz+1) reals: V + cdd phi, then rho (even rows, then odd rows)
//   DP  2nz x (ny/2 + 1): the row-pair lines of the real transforms; it shares
//       the upper half of SP, which holds nothing between the pruned inverse y
//       transform and the pruned forward one.
//   RP   ny rows x PS  real-space psi of the previous phase step (real time,
//       middle and last iterations)
//   XM, XP  ny rows x PS each: psi of planes i - 1 and i + 1 (imaginary time)
// In the middle imaginary-time iterations PP, XM and XP hold the three psi
// planes of the stencil unpadded (ny rows x nz: the stencil reads them row by
// row, consecutive threads on consecutive z), each brought in by one 1-D bulk
// copy of the contiguous plane that completes on an mbarrier.
#pragma once

#include "fused.cuh"

namespace gpe {

// Barrier of a group of NTG threads: BAR = 0 is the whole block, BAR > 0 a
// named barrier shared by the warps of one group.
template <int BAR, int NTG> __device__ __forceinline__ void group_sync() {
    if constexpr (BAR == 0)
        __syncthreads();
    else
        asm volatile("bar.sync %0, %1;" ::"n"(BAR), "n"(NTG) : "memory");
}

// All stages of a transform over a tile in shared memory, in place (each stage
// reads its butterflies into registers, synchronises, writes, synchronises).
// Element t of line b at buf[b*BS + t*TS].  NT threads of barrier group BAR
// take part (tid = index within the group).  TWS: the twiddle tables passed
// to the stages are in shared memory (plain loads instead of read-only global
// loads).
template <int SIGN, class R, int L, int COUNT, int BS, int TS, int NT, bool CMP, bool REV, bool IH = false,
          bool OH = false, int BAR = 0, bool TWS = false>
struct PlanePass {
    using C                      = cplx<R>;
    static constexpr Radices RAD = REV ? reversed(radices_of(L)) : radices_of(L);
    static constexpr int NSTG    = RAD.n;

    static constexpr int ns_before(int S) {
        int ns = 1;
        for (int s = 0; s < S; ++s)
            ns *= RAD.r[s];
        return ns;
    }

    template <int S> struct Stage {
        static constexpr int RADIX  = RAD.r[S];
        static constexpr int NS     = ns_before(S);
        static constexpr int NR     = L / RADIX;
        static constexpr int STEP   = L / (NS * RADIX);
        static constexpr int ITEMS  = COUNT * NR;
        static constexpr int ROUNDS = (ITEMS + NT - 1) / NT;
        static constexpr bool PIN   = IH && S == 0;
        static constexpr bool POUT  = OH && S == NSTG - 1;
        static_assert(!PIN || RADIX % 2 == 0, "input pruning needs an even first radix");
        static_assert(!POUT || RADIX % 2 == 0, "output pruning needs an even last radix");
        using Regs = C[ROUNDS][RADIX];

        static __device__ __forceinline__ bool valid(int it) { return ITEMS % NT == 0 || it < ITEMS; }

        // butterfly inputs (twiddled) -> DFT, in registers
        static __device__ __forceinline__ void read(const C *buf, Regs &a, const C *tw, const C *twlo,
                                                    int tid) {
#pragma unroll
            for (int rd = 0; rd < ROUNDS; ++rd) {
                const int it = rd * NT + tid;
                if (!valid(it))
                    break;
                const int j  = it / COUNT;
                const int b  = it - j * COUNT;
                const int jm = j % NS;
                const C *s   = buf + b * BS + j * TS;
#pragma unroll
                for (int k = 0; k < RADIX; ++k) {
                    if (PIN && 2 * k >= RADIX) {
                        a[rd][k] = C{(R)0, (R)0};
                        continue;
                    }
                    C v = s[k * NR * TS];
                    if (NS > 1 && k > 0) {
                        const int t = jm * k * STEP;
                        const C w   = TWS ? tw[t] : __ldg(&tw[t]);
                        if constexpr (sizeof(R) == 4 && CMP)
                            v = twmul<SIGN>(v, w, TWS ? twlo[t] : __ldg(&twlo[t]));
                        else
                            v = SIGN < 0 ? cmul(v, w) : cmulc(v, w);
                    }
                    a[rd][k] = v;
                }
                DFTZ<RADIX, SIGN, R, CMP, PIN ? RADIX / 2 : RADIX>::run(a[rd]);
            }
        }

        // stage-0 butterfly inputs straight from a loader ld(b, t) (element t of
        // line b), for a first stage that reads global memory instead of the
        // tile (no twiddles: the first stage has none)
        template <class Ld> static __device__ __forceinline__ void read_ld(Ld &ld, Regs &a, int tid) {
            static_assert(S == 0, "only the first stage reads through a loader");
#pragma unroll
            for (int rd = 0; rd < ROUNDS; ++rd) {
                const int it = rd * NT + tid;
                if (!valid(it))
                    break;
                const int j = it / COUNT;
                const int b = it - j * COUNT;
#pragma unroll
                for (int k = 0; k < RADIX; ++k)
                    a[rd][k] = (PIN && 2 * k >= RADIX) ? C{(R)0, (R)0} : ld(b, j + k * NR);
            }
#pragma unroll
            for (int rd = 0; rd < ROUNDS; ++rd) {
                if (!valid(rd * NT + tid))
                    break;
                DFTZ<RADIX, SIGN, R, CMP, PIN ? RADIX / 2 : RADIX>::run(a[rd]);
            }
        }

        static __device__ __forceinline__ void write(C *buf, const Regs &a, int tid) {
#pragma unroll
            for (int rd = 0; rd < ROUNDS; ++rd) {
                const int it = rd * NT + tid;
                if (!valid(it))
                    break;
                const int j    = it / COUNT;
                const int b    = it - j * COUNT;
                const int jm   = j % NS;
                const int idxD = (j / NS) * NS * RADIX + jm;
                C *d           = buf + b * BS + idxD * TS;
#pragma unroll
                for (int q = 0; q < RADIX; ++q)
                    if (!(POUT && 2 * q >= RADIX))
                        d[q * NS * TS] = a[rd][q];
            }
        }

        // line and element of output q of round rd
        static __device__ __forceinline__ int line(int tid, int rd) { return (rd * NT + tid) % COUNT; }
        static __device__ __forceinline__ int elem(int tid, int rd, int q) {
            const int j = (rd * NT + tid) / COUNT;
            return (j / NS) * NS * RADIX + j % NS + q * NS;
        }
    };

    template <int S, int SE> static __device__ __forceinline__ void stages(C *buf, const C *tw, const C *twlo, int tid) {
        if constexpr (S < SE) {
            typename Stage<S>::Regs a;
            Stage<S>::read(buf, a, tw, twlo, tid);
            group_sync<BAR, NT>();
            Stage<S>::write(buf, a, tid);
            group_sync<BAR, NT>();
            stages<S + 1, SE>(buf, tw, twlo, tid);
        }
    }

    using Last  = Stage<NSTG - 1>;
    using First = Stage<0>;

    // The whole transform.  The tile must be complete (caller synchronised);
    // returns after a final synchronisation.
    static __device__ __forceinline__ void run(C *buf, const C *tw, const C *twlo, int tid) {
        stages<0, NSTG>(buf, tw, twlo, tid);
    }
    // All stages, the last one handing its outputs to st(b, t, v) (element t of
    // line b) instead of writing the tile.  Other threads may still read the
    // tile on return: synchronise before reusing it.
    template <int S0 = 0, class St>
    static __device__ __forceinline__ void run_emit(C *buf, St st, const C *tw, const C *twlo, int tid) {
        stages<S0, NSTG - 1>(buf, tw, twlo, tid);
        typename Last::Regs a;
        Last::read(buf, a, tw, twlo, tid);
#pragma unroll
        for (int rd = 0; rd < Last::ROUNDS; ++rd) {
            if (!Last::valid(rd * NT + tid))
                break;
            const int b = Last::line(tid, rd);
#pragma unroll
            for (int q = 0; q < Last::RADIX; ++q)
                if (!(Last::POUT && 2 * q >= Last::RADIX))
                    st(b, Last::elem(tid, rd, q), a[rd][q]);
        }
    }
    // All stages but the writes of the last one: a = outputs of the last stage,
    // Last::line / Last::elem give their positions.  Other threads may still
    // read the tile: synchronise before writing it.
    static __device__ __forceinline__ void run_to_regs(C *buf, typename Last::Regs &a, const C *tw,
                                                       const C *twlo, int tid) {
        stages<0, NSTG - 1>(buf, tw, twlo, tid);
        Last::read(buf, a, tw, twlo, tid);
    }
    // Starts from the first stage's inputs in registers, laid out as
    // run_to_regs of the reversed transform leaves them (same thread mapping).
    // The tile must be free (caller synchronised).
    static __device__ __forceinline__ void run_from_regs(C *buf, typename First::Regs &a, const C *tw,
                                                         const C *twlo, int tid) {
        static_assert(First::NS == 1, "first stage");
#pragma unroll
        for (int rd = 0; rd < First::ROUNDS; ++rd) {
            if (!First::valid(rd * NT + tid))
                break;
            DFT<First::RADIX, SIGN, R, CMP>::run(a[rd]);
        }
        First::write(buf, a, tid);
        group_sync<BAR, NT>();
        stages<1, NSTG>(buf, tw, twlo, tid);
    }
};

// Stages [S, SE) of in-place pass P on pbuf run jointly with stages [T, TE)
// of pass Q on qbuf: stage S+k of P and T+k of Q read together, share the
// barrier, write together.  Two independent butterflies per thread and half
// the barriers of running the passes one after the other.
template <class P, int S, int SE, class Q, int T, int TE, class C>
__device__ __forceinline__ void joint_stages(C *pbuf, const C *ptw, const C *ptl, C *qbuf, const C *qtw,
                                             const C *qtl, int tid) {
    constexpr bool DP = S < SE, DQ = T < TE;
    if constexpr (DP || DQ) {
        using SP_ = typename P::template Stage<DP ? S : 0>;
        using SQ_ = typename Q::template Stage<DQ ? T : 0>;
        typename SP_::Regs pa;
        typename SQ_::Regs qa;
        if constexpr (DP)
            SP_::read(pbuf, pa, ptw, ptl, tid);
        if constexpr (DQ)
            SQ_::read(qbuf, qa, qtw, qtl, tid);
        __syncthreads();
        if constexpr (DP)
            SP_::write(pbuf, pa, tid);
        if constexpr (DQ)
            SQ_::write(qbuf, qa, tid);
        __syncthreads();
        joint_stages<P, S + 1, SE, Q, T + 1, TE>(pbuf, ptw, ptl, qbuf, qtw, qtl, tid);
    }
}

struct YZTwid {
    Twid ky, kz, dy, dz;
};

// ROWS x COLS plane (contiguous in global) -> shared rows of stride PS, by
// cp.async (no register staging)
template <class T, int ROWS, int COLS, int PS, int NT>
__device__ __forceinline__ void plane_in_async(T *dst, const T *src, int tid) {
    static_assert(sizeof(T) == 8 || sizeof(T) == 4, "8- or 4-byte elements");
#pragma unroll 4
    for (int e = tid; e < ROWS * COLS; e += NT) {
        const int r = e / COLS, k = e - r * COLS;
        if constexpr (sizeof(T) == 8)
            cp_async8(&dst[r * PS + k], &src[e]);
        else
            cp_async4(&dst[r * PS + k], &src[e]);
    }
}

// Global plane (ROWS x COLS complex, contiguous) <-> shared tile with row stride
// PS.  Each thread issues all its 16-byte loads before any shared store.
template <class R, int ROWS, int COLS, int PS, int NT>
__device__ __forceinline__ void plane_in(cplx<R> *__restrict__ dst, const cplx<R> *__restrict__ src, int tid) {
    using C          = cplx<R>;
    static_assert(COLS % 2 == 0 && sizeof(C) == 8, "pairs of complex64 per 16-byte load");
    constexpr int N2 = ROWS * COLS / 2;
    constexpr int PER = (N2 + NT - 1) / NT;
    const float4 *s4 = reinterpret_cast<const float4 *>(src);
    float4 v[PER];
#pragma unroll
    for (int u = 0; u < PER; ++u) {
        const int e = u * NT + tid;
        if (N2 % NT == 0 || e < N2)
            v[u] = __ldg(&s4[e]);
    }
#pragma unroll
    for (int u = 0; u < PER; ++u) {
        const int e = u * NT + tid;
        if (N2 % NT == 0 || e < N2) {
            const int r = (2 * e) / COLS, k = 2 * e - r * COLS;
            dst[r * PS + k]     = C{v[u].x, v[u].y};
            dst[r * PS + k + 1] = C{v[u].z, v[u].w};
        }
    }
}
template <class R, int ROWS, int COLS, int PS, int NT>
__device__ __forceinline__ void plane_out(cplx<R> *__restrict__ dst, const cplx<R> *__restrict__ src, int tid) {
    static_assert(COLS % 2 == 0 && sizeof(cplx<R>) == 8, "pairs of complex64 per 16-byte store");
    constexpr int N2 = ROWS * COLS / 2;
    float4 *d4       = reinterpret_cast<float4 *>(dst);
#pragma unroll 4
    for (int e = tid; e < N2; e += NT) {
        const int r = (2 * e) / COLS, k = 2 * e - r * COLS;
        const cplx<R> a = src[r * PS + k], b = src[r * PS + k + 1];
        d4[e]           = make_float4(a.x, a.y, b.x, b.y);
    }
}

// Plane-kernel geometry for ny = NY, nz = NZ.
template <class R, int NY, int NZ> struct YZShape {
    using C                      = cplx<R>;
    static constexpr int PS      = NZ + 1;           // complex row stride of SP, PP
    static constexpr int FS      = NZ + 1;           // real row stride of FP
    static constexpr int NP      = NY / 2;           // row pairs
    static constexpr int LD      = 2 * NZ;           // real-transform line length
    static constexpr int TD      = NP + 1;           // DP element stride
    static constexpr bool ALIAS  = LD * TD <= NY * PS; // DP fits in the upper half of SP
    static constexpr size_t SP_B = sizeof(C) * 2 * NY * PS;
    static constexpr size_t PP_B = sizeof(C) * NY * PS;
    // FP keeps even rows and odd rows in two halves, the odd half starting 16
    // banks further on: lanes of consecutive rows, and lanes of consecutive row
    // pairs, then fall in distinct banks (FS odd)
    static constexpr int FH      = NP * FS + (((16 - (NP * FS) % 32) % 32) + 32) % 32;
    static constexpr int FPN     = FH + NP * FS;     // floats in FP
    static constexpr size_t FP_B = sizeof(R) * FPN;
    static __device__ __forceinline__ int fpi(int r, int k) { return (r & 1) * FH + (r >> 1) * FS + k; }
    static constexpr size_t DP_B = ALIAS ? 0 : sizeof(C) * LD * TD;
    static constexpr size_t SMEM = SP_B + PP_B + FP_B + DP_B; // imaginary time, RT prologue
    static constexpr size_t RP_B = sizeof(C) * NY * PS;
    static constexpr size_t SMEM_RT = SMEM + RP_B;            // RT middle and last iterations
    static constexpr size_t SMEM_IT = SMEM + 2 * RP_B;        // IT: the two x-neighbour planes
    template <int MODE> static constexpr size_t smem_base() {
        return (MODE == ZM_RT_MID || MODE == ZM_RT_EPI) ? SMEM_RT : (MODE == ZM_IT_MID ? SMEM_IT : SMEM);
    }
    // The twiddle tables, staged in shared memory behind the tiles (TW): the
    // dipolar y (2ny) and z (2nz) lines, the kinetic y (ny) and z (nz) lines
    // with their rounding remainders.  One SM runs one plane per launch, so its
    // L1 holds none of them at kernel start: read from global memory, every
    // stage's first twiddle loads would wait for L2.
    static constexpr int TW_DY = 0, TW_DZ = 2 * NY, TW_KY = TW_DZ + LD, TW_KYL = TW_KY + NY,
                         TW_KZ = TW_KYL + NY, TW_KZL = TW_KZ + NZ, TWN = TW_KZL + NZ;
    static constexpr size_t TW_B = sizeof(C) * TWN;
    static_assert(SMEM % 8 == 0 && SMEM_RT % 8 == 0 && SMEM_IT % 8 == 0, "8-byte aligned twiddle region");
    template <int MODE> static constexpr size_t smem() { return smem_base<MODE>() + TW_B; }
    // cp.async of the tables into TW (the kinetic ones only in real time)
    template <bool KIN>
    static __device__ __forceinline__ void twiddles_in(C *TW, const YZTwid &tw, int tid, int nt) {
        auto cp = [&](int off, const void *src, int n) {
            for (int e = tid; e < n; e += nt)
                cp_async8(&TW[off + e], reinterpret_cast<const C *>(src) + e);
        };
        cp(TW_DY, tw.dy.tw, 2 * NY);
        cp(TW_DZ, tw.dz.tw, LD);
        if (KIN) {
            cp(TW_KY, tw.ky.tw, NY);
            cp(TW_KYL, tw.ky.lo, NY);
            cp(TW_KZ, tw.kz.tw, NZ);
            cp(TW_KZL, tw.kz.lo, NZ);
        }
    }
    // the same tables as kernel arguments pointing into TW (the dipolar
    // remainders are not used: those transforms apply plain twiddles)
    static __device__ __forceinline__ YZTwid shared_twiddles(const C *TW, const YZTwid &tw) {
        YZTwid t = tw;
        t.dy.tw  = TW + TW_DY;
        t.dz.tw  = TW + TW_DZ;
        t.ky     = Twid{TW + TW_KY, TW + TW_KYL};
        t.kz     = Twid{TW + TW_KZ, TW + TW_KZL};
        return t;
    }
    static constexpr int NT0     = 2 * NY * NZ / 16;
    static constexpr int NT      = NT0 < 128 ? 128 : (NT0 > 512 ? 512 : (NT0 + 31) / 32 * 32);
    // Threads of the kernel in each mode: the imaginary-time modes (62-80
    // registers, no kinetic chain; latency bound on their plane loads) run twice
    // the real-time count, at most 1024.
    // WIDE = false keeps the real-time count in imaginary time too: the
    // autotuner picks per grid (the wide block wins at 64^2 x 16, the narrow
    // one at 128^2 x 32)
    template <int MODE, bool WIDE = true> static constexpr int nt() {
        return (WIDE && (MODE == ZM_IT_PRO || MODE == ZM_IT_MID)) ? (2 * NT > 1024 ? 1024 : 2 * NT) : NT;
    }
};

// The dipolar chain of a plane, run by NTG threads of barrier group BAR.
template <class R, int NY, int NZ, int NTG, int BAR, bool TWS = false> struct DipolarPlane {
    using C         = cplx<R>;
    using G         = YZShape<R, NY, NZ>;
    static constexpr int PS = G::PS, FS = G::FS, NP = G::NP, LD = G::LD, TD = G::TD;

    // iFFT_y(2ny, lower half kept) of SP, C2R_z of the row pairs -> FP = V + cdd
    // phi (FP holds V on entry), and phi -> global when WRITE_PHI.  SP must be
    // loaded (caller synchronised); the caller's other cp.async group (psi, V)
    // is waited for here, overlapped with the y transforms.
    // S_g: the plane of the spectrum in global memory, read by the first stage
    // of the y transform (which writes SP)
    template <bool WRITE_PHI>
    static __device__ __forceinline__ void inverse(const C *S_g, C *SP, C *DP, R *FP, R *phi_g, R cdd,
                                                   const YZTwid &tw, int t) {
        using DYI = PlanePass<+1, R, 2 * NY, NZ, 1, PS, NTG, false, true, false, true, BAR, TWS>;
        {
            auto lds = [&](int b, int r) { return S_g[r * NZ + b]; };
            typename DYI::First::Regs a0;
            DYI::First::read_ld(lds, a0, t);
            DYI::First::write(SP, a0, t);
            group_sync<BAR, NTG>();
        }
        DYI::template stages<1, DYI::NSTG>(SP, (const C *)tw.dy.tw, (const C *)tw.dy.lo, t);
        cp_async_wait<0>(); // visible to the block after the next barrier
        // pair lines: z[m] = X_a[m] + i X_b[m] over the full 2nz-point spectrum
        // (bins 1..nz stored at kz - 1, bin 0 is zero, bins > nz by symmetry);
        // DP may share SP's upper half (rows >= NY), which nothing reads any more.
        // Consecutive threads take consecutive m: SP rows read contiguously.
        for (int e = t; e < NP * LD; e += NTG) {
            const int m = e % LD, p = e / LD;
            C z         = C{(R)0, (R)0};
            if (m > 0) {
                const int mm = m <= NZ ? m : LD - m;
                const C xa   = SP[(2 * p) * PS + mm - 1];
                const C xb   = SP[(2 * p + 1) * PS + mm - 1];
                if (m == NZ)
                    z = C{xa.x, xb.x}; // self-conjugate bin: real parts only
                else if (m < NZ)
                    z = C{xa.x - xb.y, xa.y + xb.x};
                else
                    z = C{xa.x + xb.y, xb.x - xa.y};
            }
            DP[p + m * TD] = z;
        }
        group_sync<BAR, NTG>();
        PlanePass<+1, R, LD, NP, 1, TD, NTG, false, true, false, true, BAR, TWS>::run(
            DP, (const C *)tw.dz.tw, (const C *)tw.dz.lo, t);
        for (int e = t; e < NY * NZ; e += NTG) {
            const int r = e / NZ, k = e - r * NZ;
            const C zz  = DP[(r >> 1) + k * TD];
            const R f   = (r & 1) ? zz.y : zz.x;
            if (WRITE_PHI)
                phi_g[e] = f;
            FP[G::fpi(r, k)] += cdd * f;
        }
    }

    // Row pair p of rho (FP): element m of its complex line (m < nz; the upper
    // half of the zero-padded line is zero and never read).  Consecutive p at
    // the odd stride FS: distinct banks.
    static __device__ __forceinline__ C rho_pair(const R *FP, int p, int m) {
        return C{FP[G::fpi(2 * p, m)], FP[G::fpi(2 * p + 1, m)]};
    }
    // Row r, bin m (1 <= m <= nz) of the real transform of rho, unpacked from
    // the spectrum Z of its row pair in DP: (Z_m + conj(Z_{L-m}))/2 for the even
    // row, (Z_m - conj(Z_{L-m}))/(2i) for the odd one.  Consecutive m at the odd
    // stride TD: distinct banks.
    static __device__ __forceinline__ C rho_bin(const C *DP, int r, int m) {
        const int p = r >> 1;
        const C zm  = DP[p + m * TD];
        const C zc  = DP[p + (LD - m) * TD];
        if ((r & 1) == 0)
            return C{(R)0.5 * (zm.x + zc.x), (R)0.5 * (zm.y - zc.y)};
        return C{(R)0.5 * (zm.y + zc.y), (R)0.5 * (zc.x - zm.x)};
    }

    // rho (FP) -> R2C_z of the row pairs -> FFT_y(2ny, upper half zero) -> S (global).
    // FP must be complete and DP free (caller synchronised).  The first stage of
    // the R2C reads the row pairs from FP, the first stage of the y transform
    // unpacks the rows' bins from DP: neither goes through a copy in the tiles.
    static __device__ __forceinline__ void forward(C *SP, C *DP, const R *FP, C *S_g, const YZTwid &tw, int t) {
        using R2C = PlanePass<-1, R, LD, NP, 1, TD, NTG, false, false, true, false, BAR, TWS>;
        using DYF = PlanePass<-1, R, 2 * NY, NZ, 1, PS, NTG, false, false, true, false, BAR, TWS>;
        {
            auto ldr = [&](int p, int m) { return rho_pair(FP, p, m); };
            typename R2C::First::Regs a0;
            R2C::First::read_ld(ldr, a0, t);
            R2C::First::write(DP, a0, t);
            group_sync<BAR, NTG>();
        }
        R2C::template stages<1, R2C::NSTG>(DP, (const C *)tw.dz.tw, (const C *)tw.dz.lo, t);
        {
            // bins 1..nz of the rows, stored at kz - 1 (line b = kz - 1)
            auto ldu = [&](int b, int r) { return rho_bin(DP, r, b + 1); };
            typename DYF::First::Regs a0;
            DYF::First::read_ld(ldu, a0, t);
            group_sync<BAR, NTG>(); // DP (SP's upper half) read by every thread
            DYF::First::write(SP, a0, t);
            group_sync<BAR, NTG>();
        }
        static_assert(DYF::NSTG >= 2, "y lines of at least two stages");
        DYF::template run_emit<1>(
            SP, [&](int b, int r, C v) { S_g[r * NZ + b] = v; }, (const C *)tw.dy.tw, (const C *)tw.dy.lo, t);
    }
};

template <class R, int NY, int NZ, int MODE, bool WIDE = true>
__global__ void __launch_bounds__(YZShape<R, NY, NZ>::template nt<MODE, WIDE>()) k4_yz(ZArgs a, YZTwid tw) {
    using C                = cplx<R>;
    using G                = YZShape<R, NY, NZ>;
    constexpr int NT       = G::template nt<MODE, WIDE>();
    constexpr int PS       = G::PS;
    constexpr bool RT      = MODE <= ZM_RT_EPI;
    constexpr bool HAS_INV = (MODE == ZM_RT_MID || MODE == ZM_RT_EPI || MODE == ZM_IT_MID);
    const int tid          = threadIdx.x;
    const int i            = blockIdx.x; // x plane
    const int nx           = a.nx;

    C *SP  = reinterpret_cast<C *>(g_smem);
    C *PP  = SP + 2 * NY * PS;
    R *FP  = reinterpret_cast<R *>(PP + NY * PS);
    C *DP  = G::ALIAS ? SP + NY * PS : reinterpret_cast<C *>(FP + G::FPN);
    C *RP  = reinterpret_cast<C *>(g_smem + G::SMEM); // RT middle and last iterations only
    C *XM  = RP;                                      // IT: x-neighbour planes
    C *XP  = RP + NY * PS;
    __shared__ double red[NT / 32];

    C *S_g         = reinterpret_cast<C *>(a.S) + (size_t)i * 2 * NY * NZ;
    const R *V_g   = reinterpret_cast<const R *>(a.V) + (size_t)i * NY * NZ;
    R *phi_g       = reinterpret_cast<R *>(a.phi) + (size_t)i * NY * NZ;
    C *P_o         = reinterpret_cast<C *>(a.psi_out) + (size_t)i * NY * NZ;
    C *Pr_g        = reinterpret_cast<C *>(a.psi_r) + (size_t)i * NY * NZ;
    const R cdd    = (R)a.cdd;

    // The step coefficients, read first: the chunk counter and the table entry
    // it selects are two dependent L2 reads, which land behind the plane loads
    // instead of stalling every warp at the phase step (real time: the sum of
    // this iteration's and the next one's half steps in the middle iterations;
    // imaginary time: the table's first entry).
    R g3 = (R)0, gw = (R)0;
    {
        const StepCoef c0 = a.step.coef[RT ? *a.step.base + a.step.local : 0];
        if (MODE == ZM_RT_MID) {
            const StepCoef c1 = a.step.coef[*a.step.base + a.step.local + 1];
            g3                = (R)(c0.g3w + c1.g3w);
            gw                = (R)(c0.gw15 + c1.gw15);
        } else {
            g3 = (R)c0.g3w;
            gw = (R)c0.gw15;
        }
    }

    // Imaginary time: the kept boundary values of this thread's stencil points,
    // also read at kernel start (every row has its two z-boundary points, so
    // read at the stencil step they would hold every warp for an L2 round trip)
    constexpr int SE = (NY * NZ + NT - 1) / NT; // stencil points per thread
    C bpre[MODE == ZM_IT_MID ? SE : 1];
    if constexpr (MODE == ZM_IT_MID) {
        const C *bp     = reinterpret_cast<const C *>(a.bnd) + (size_t)i * NY * NZ;
        const bool xin0 = i >= 1 && i < nx - 1;
#pragma unroll
        for (int j = 0; j < SE; ++j) {
            const int e = tid + j * NT;
            const int r = e / NZ, k = e - r * NZ;
            if (e < NY * NZ && (!xin0 || r < 1 || r >= NY - 1 || k < 1 || k >= NZ - 1))
                bpre[j] = __ldg(&bp[e]);
        }
    }

    // ---- load the planes (cp.async groups: none; psi and V; kept real-space psi) ---
    // In real time with the inverse transforms (middle and last iterations) the
    // first stages of the inverse y transforms read the S and psi planes from
    // global memory themselves (RT_DIRECT below): the tile is written once, by
    // those stages, instead of by the copy and again by them.
    // (In imaginary time the dipolar inverse's first stage reads the S plane
    // from global memory the same way.)
    constexpr bool RT_DIRECT = RT && HAS_INV;
    constexpr bool IT_BULK   = MODE == ZM_IT_MID; // the stencil's planes by bulk copies
    __shared__ __align__(8) unsigned long long pbar;
    // twiddle tables first (cp.async group 0): they land long before the
    // first stage's plane loads, and no stage waits for L2 on a twiddle
    C *TW = reinterpret_cast<C *>(g_smem + G::template smem_base<MODE>());
    G::template twiddles_in<RT>(TW, tw, tid, NT);
    const YZTwid tws = G::shared_twiddles(TW, tw);
    cp_async_commit();
    if (RT && !RT_DIRECT)
        plane_in_async<C, NY, NZ, PS, NT>(PP, reinterpret_cast<const C *>(a.psi_in) + (size_t)i * NY * NZ, tid);
    if (MODE != ZM_IT_PRO) {
#pragma unroll 4
        for (int e = tid; e < NY * NZ; e += NT) {
            const int r = e / NZ, k = e - r * NZ;
            cp_async4(&FP[G::fpi(r, k)], &V_g[e]);
        }
    }
    if (IT_BULK && tid == 0) {
        // psi of this plane and (interior planes) of its two x neighbours:
        // three contiguous 8 ny nz-byte blocks, one bulk copy each
        const C *pin      = reinterpret_cast<const C *>(a.psi_in);
        const bool inner  = i >= 1 && i < nx - 1;
        const unsigned pb = (unsigned)(sizeof(C) * NY * NZ);
        mbar_init(&pbar, 1);
        mbar_expect_tx(&pbar, inner ? 3 * pb : pb);
        bulk_g2s(PP, pin + (size_t)i * NY * NZ, pb, &pbar);
        if (inner) {
            bulk_g2s(XM, pin + (size_t)(i - 1) * NY * NZ, pb, &pbar);
            bulk_g2s(XP, pin + (size_t)(i + 1) * NY * NZ, pb, &pbar);
        }
    }
    cp_async_commit();
    constexpr bool KEPT = MODE == ZM_RT_MID || MODE == ZM_RT_EPI;
    if (KEPT) {
        // needed only at the phase step: waited for there, behind the transforms;
        // V (the group before) is waited for before the C2R's stages
        plane_in_async<C, NY, NZ, PS, NT>(RP, Pr_g, tid);
        cp_async_commit();
    } else if (HAS_INV && !RT) {
        cp_async_wait<1>(); // S; psi and V are waited for inside the dipolar inverse
    } else {
        cp_async_wait<0>();
    }
    __syncthreads();

    if constexpr (RT) {
        // The dipolar and the kinetic transforms run stage by stage side by side
        // (joint_stages); they meet for phi before the phase and rho after it.
        constexpr int NP = G::NP, LD = G::LD, TD = G::TD;
        using DYI = PlanePass<+1, R, 2 * NY, NZ, 1, PS, NT, false, true, false, true, 0, true>;
        using KYI = PlanePass<+1, R, NY, NZ, 1, PS, NT, true, false, false, false, 0, true>;
        using C2R = PlanePass<+1, R, LD, NP, 1, TD, NT, false, true, false, true, 0, true>;
        using ZI  = PlanePass<+1, R, NZ, NY, PS, 1, NT, true, false, false, false, 0, true>;
        using ZF  = PlanePass<-1, R, NZ, NY, PS, 1, NT, true, true, false, false, 0, true>;
        using R2C = PlanePass<-1, R, LD, NP, 1, TD, NT, false, false, true, false, 0, true>;
        using KYF = PlanePass<-1, R, NY, NZ, 1, PS, NT, true, false, false, false, 0, true>;
        using DYF = PlanePass<-1, R, 2 * NY, NZ, 1, PS, NT, false, false, true, false, 0, true>;
        static_assert(ZI::Last::RADIX == ZF::First::RADIX && ZI::Last::ROUNDS == ZF::First::ROUNDS &&
                          ZI::Last::ITEMS == ZF::First::ITEMS,
                      "paired z transforms share the register layout");
        static_assert(KYF::NSTG >= 2 && DYF::NSTG >= 2, "y lines of at least two stages");
        const C *dyt = (const C *)tws.dy.tw, *dyl = (const C *)tws.dy.lo;
        const C *dzt = (const C *)tws.dz.tw, *dzl = (const C *)tws.dz.lo;
        const C *kyt = (const C *)tws.ky.tw, *kyl = (const C *)tws.ky.lo;
        const C *kzt = (const C *)tws.kz.tw, *kzl = (const C *)tws.kz.lo;
        constexpr bool WRITE_PHI = MODE != ZM_RT_MID; // read only after the last iteration
        typename ZI::Last::Regs zr;
        if (HAS_INV) {
            // dipolar iFFT_y (lower half kept) || kinetic iFFT_y; their first
            // stages load the planes from global memory (coalesced along the
            // nz columns) and write the tiles
            {
                const C *Q_g = reinterpret_cast<const C *>(a.psi_in) + (size_t)i * NY * NZ;
                auto lds     = [&](int b, int t) { return S_g[t * NZ + b]; };
                auto ldq     = [&](int b, int t) { return Q_g[t * NZ + b]; };
                typename DYI::First::Regs da0;
                typename KYI::First::Regs ka0;
                DYI::First::read_ld(lds, da0, tid);
                KYI::First::read_ld(ldq, ka0, tid);
                DYI::First::write(SP, da0, tid);
                KYI::First::write(PP, ka0, tid);
                cp_async_wait<2>(); // the twiddles (V and the kept psi may still be in flight)
                __syncthreads();
            }
            joint_stages<DYI, 1, DYI::NSTG, KYI, 1, KYI::NSTG>(SP, dyt, dyl, PP, kyt, kyl, tid);
            // C2R pair lines: z[m] = X_a[m] + i X_b[m] over the full 2nz-point
            // spectrum (bins 1..nz stored at kz - 1, bin 0 zero, bins > nz by
            // symmetry); DP shares SP's upper half, which holds nothing now;
            // consecutive threads take consecutive m (SP rows read contiguously)
            for (int e = tid; e < NP * LD; e += NT) {
                const int m = e % LD, p = e / LD;
                C z         = C{(R)0, (R)0};
                if (m > 0) {
                    const int mm = m <= NZ ? m : LD - m;
                    const C xa   = SP[(2 * p) * PS + mm - 1];
                    const C xb   = SP[(2 * p + 1) * PS + mm - 1];
                    if (m == NZ)
                        z = C{xa.x, xb.x}; // self-conjugate bin: real parts only
                    else if (m < NZ)
                        z = C{xa.x - xb.y, xa.y + xb.x};
                    else
                        z = C{xa.x + xb.y, xb.x - xa.y};
                }
                DP[p + m * TD] = z;
            }
            if (KEPT)
                cp_async_wait<1>(); // V: visible to the block after the barriers below
            __syncthreads();
            // C2R || kinetic iFFT_z, all stages but the last
            joint_stages<C2R, 0, C2R::NSTG - 1, ZI, 0, ZI::NSTG - 1>(DP, dzt, dzl, PP, kzt, kzl, tid);
            {
                // last C2R stage -> FP = V + cdd phi; last iFFT_z stage -> registers
                typename C2R::Last::Regs ca;
                C2R::Last::read(DP, ca, dzt, dzl, tid);
                ZI::Last::read(PP, zr, kzt, kzl, tid);
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
                        if (WRITE_PHI) {
                            phi_g[(2 * p) * NZ + k]     = v.x;
                            phi_g[(2 * p + 1) * NZ + k] = v.y;
                        }
                    }
                }
            }
        } else {
            // prologue: phi of the previous calc_fi3d
            for (int e = tid; e < NY * NZ; e += NT) {
                const int r = e / NZ, k = e - r * NZ;
                FP[G::fpi(r, k)] += cdd * phi_g[e];
            }
        }
        if (KEPT)
            cp_async_wait<0>(); // RP, visible to the block after the barrier
        __syncthreads(); // FP = V + cdd phi

        // merged potential half steps: theta = -dt/2 [cV (V + cdd phi) + g3 |psi|^2 + gw |psi|^3]
        // (g3, gw: the step coefficients loaded at kernel start)
        const R cV = MODE == ZM_RT_MID ? (R)2 : (R)1;
        const R hdt = (R)a.half_dt, wat = (R)a.w_atoms;
        const bool xin = i >= 1 && i < nx - 1;
        auto phase = [&](C p, int y, int z) -> C {
            const int f = G::fpi(y, z);
            if (xin && y >= 1 && y < NY - 1 && z >= 1 && z < NZ - 1) {
                const R dens  = p.x * p.x + p.y * p.y;
                const R am    = sqrt(dens);
                const R total = cV * FP[f] + g3 * dens + gw * (am * am * am);
                R s, c;
                sincos_r<R>((R)-0.5 * hdt * total, &s, &c);
                p = apply_wm1(p, C{(R)-2 * s * s, (R)2 * s * c});
            }
            FP[f] = wat * (p.x * p.x + p.y * p.y); // rho for the next dipolar spectrum
            return p;
        };
        if (MODE == ZM_RT_PRO) {
            // psi is in real space; the plane after the phase is kept in psi_r
            for (int e = tid; e < NY * NZ; e += NT) {
                const int r = e / NZ, k = e - r * NZ;
                const C v      = phase(PP[r * PS + k], r, k);
                PP[r * PS + k] = v;
                Pr_g[e]        = v;
            }
        } else {
#pragma unroll
            for (int rd = 0; rd < ZI::Last::ROUNDS; ++rd) {
                if (!ZI::Last::valid(rd * NT + tid))
                    break;
                const int y = ZI::Last::line(tid, rd);
#pragma unroll
                for (int q = 0; q < ZI::Last::RADIX; ++q) {
                    const int z = ZI::Last::elem(tid, rd, q);
                    // psi = kept psi + kinetic increment, then the phase step;
                    // the new psi goes back to RP (stored coalesced further on)
                    zr[rd][q] = phase(cadd(zr[rd][q], RP[y * PS + z]), y, z);
                    if (MODE == ZM_RT_MID)
                        RP[y * PS + z] = zr[rd][q];
                }
            }
            if (MODE == ZM_RT_EPI) {
                // psi in real space -> global (the last z reads of PP are behind a barrier)
                ZI::Last::write(PP, zr, tid);
                __syncthreads();
                plane_out<R, NY, NZ, PS, NT>(P_o, PP, tid);
                return;
            }
        }
        __syncthreads(); // rho complete

        using DW = DipolarPlane<R, NY, NZ, NT, 0, true>;
        if (MODE == ZM_RT_PRO) {
            // R2C pair lines from rho (upper half zero) || kinetic FFT_z
            for (int e = tid; e < NP * NZ; e += NT) {
                const int m = e % NZ, p = e / NZ;
                DP[p + m * TD] = DW::rho_pair(FP, p, m);
            }
            __syncthreads();
            joint_stages<R2C, 0, R2C::NSTG, ZF, 0, ZF::NSTG>(DP, dzt, dzl, PP, kzt, kzl, tid);
        } else {
            // first FFT_z stage from the registers (the iFFT_z reads of PP are
            // behind the two barriers above) || first R2C stage reading the row
            // pairs of rho from FP (DP, SP's upper half, is free since the C2R)
#pragma unroll
            for (int rd = 0; rd < ZF::First::ROUNDS; ++rd) {
                if (!ZF::First::valid(rd * NT + tid))
                    break;
                DFT<ZF::First::RADIX, -1, R, true>::run(zr[rd]);
            }
            ZF::First::write(PP, zr, tid);
            {
                auto ldr = [&](int p, int m) { return DW::rho_pair(FP, p, m); };
                typename R2C::First::Regs ra;
                R2C::First::read_ld(ldr, ra, tid);
                R2C::First::write(DP, ra, tid);
            }
            __syncthreads();
            plane_out<R, NY, NZ, PS, NT>(Pr_g, RP, tid); // kept psi for the next iteration
            joint_stages<R2C, 1, R2C::NSTG, ZF, 1, ZF::NSTG>(DP, dzt, dzl, PP, kzt, kzl, tid);
        }
        // first stages of the forward y transforms: the dipolar one unpacks the
        // rows' bins from the R2C output in DP || the kinetic one reads PP
        {
            using K0 = typename KYF::template Stage<0>;
            typename K0::Regs ka;
            K0::read(PP, ka, kyt, kyl, tid);
            typename DYF::First::Regs da;
            auto ldu = [&](int b, int r) { return DW::rho_bin(DP, r, b + 1); };
            DYF::First::read_ld(ldu, da, tid);
            __syncthreads(); // DP (SP's upper half) and PP read by every thread
            K0::write(PP, ka, tid);
            DYF::First::write(SP, da, tid);
            __syncthreads();
        }
        // dipolar FFT_y (upper half zero) || kinetic FFT_y, the last stages
        // storing straight to global memory
        joint_stages<DYF, 1, DYF::NSTG - 1, KYF, 1, KYF::NSTG - 1>(SP, dyt, dyl, PP, kyt, kyl, tid);
        {
            typename DYF::Last::Regs da;
            DYF::Last::read(SP, da, dyt, dyl, tid);
#pragma unroll
            for (int rd = 0; rd < DYF::Last::ROUNDS; ++rd) {
                if (!DYF::Last::valid(rd * NT + tid))
                    break;
                const int b = DYF::Last::line(tid, rd);
#pragma unroll
                for (int q = 0; q < DYF::Last::RADIX; ++q)
                    S_g[DYF::Last::elem(tid, rd, q) * NZ + b] = da[rd][q];
            }
        }
        {
            typename KYF::Last::Regs kb;
            KYF::Last::read(PP, kb, kyt, kyl, tid);
#pragma unroll
            for (int rd = 0; rd < KYF::Last::ROUNDS; ++rd) {
                if (!KYF::Last::valid(rd * NT + tid))
                    break;
                const int b = KYF::Last::line(tid, rd);
#pragma unroll
                for (int q = 0; q < KYF::Last::RADIX; ++q)
                    P_o[KYF::Last::elem(tid, rd, q) * NZ + b] = kb[rd][q];
            }
        }
    } else {
        using DW = DipolarPlane<R, NY, NZ, NT, 0, true>;
        // imaginary time: psi_in / sqrt(divisor)
        const C *__restrict__ pin = reinterpret_cast<const C *>(a.psi_in);
        C *__restrict__ pout      = reinterpret_cast<C *>(a.psi_out);
        const R sc        = (R)(1.0 / sqrt(a.norm_state[1]));
        const R wat       = (R)a.w_atoms;
        const size_t pln  = (size_t)NY * NZ;
        const size_t base = (size_t)i * pln;
        double acc        = 0.0;
        if (MODE == ZM_IT_PRO) {
            for (int e = tid; e < NY * NZ; e += NT) {
                const int r = e / NZ, k = e - r * NZ;
                const C p   = __ldg(&pin[base + e]);
                FP[G::fpi(r, k)] = wat * (p.x * p.x + p.y * p.y);
            }
        } else {
            DW::template inverse<true>(S_g, SP, DP, FP, phi_g, cdd, tws, tid);
            __syncthreads(); // FP complete
            const R g3w = g3, gw15 = gw; // a.step.coef[0], loaded at kernel start
            const R cx = (R)a.cx, cy = (R)a.cy, cz = (R)a.cz, dtau = (R)a.dtau;
            const bool xin = i >= 1 && i < nx - 1;
            // the three planes (bulk copies issued at kernel start); a copy that
            // has not landed after the bounded wait is reported in status[1]
            if (!mbar_wait(&pbar, 0, 1 << 22)) {
                a.status[1] = 1;
                mbar_wait(&pbar, 0, 1 << 22);
            }
#pragma unroll
            for (int j = 0; j < SE; ++j) {
                const int e = tid + j * NT;
                if (SE * NT != NY * NZ && e >= NY * NZ)
                    break;
                const int r = e / NZ, k = e - r * NZ;
                const size_t q = base + e;
                C o;
                if (!xin || r < 1 || r >= NY - 1 || k < 1 || k >= NZ - 1) {
                    o = bpre[j]; // bnd[q], read at kernel start
                } else {
                    const C *pp = PP + e; // this plane and its x neighbours (unpadded)
                    const C c0 = cscale(pp[0], sc);
                    const C xm = cscale(XM[e], sc), xp = cscale(XP[e], sc);
                    const C ym = cscale(pp[-NZ], sc), yp = cscale(pp[NZ], sc);
                    const C zm = cscale(pp[-1], sc), zp = cscale(pp[1], sc);
                    const R vv   = FP[G::fpi(r, k)];
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
                FP[G::fpi(r, k)] = wat * (o.x * o.x + o.y * o.y);
            }
        }
        __syncthreads(); // rho complete; SP's upper half (DP) free
        DW::forward(SP, DP, FP, S_g, tws, tid);

        // ---- norm of psi' (imaginary time): deterministic two-level reduction -----
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
}

} // namespace gpe
