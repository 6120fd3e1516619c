// Compile-time block FFT (line length, tile shape and thread count fixed at
// compile time, so that every index division folds into shifts and multiplies
// and every stage loop unrolls).
//
// Tile layout as in fft_block.cuh: COUNT lines of length L, element t of line b
// at s[b + t*TS] (TS >= COUNT).  Stages are the mixed-radix Stockham auto-sort
// of fft_block.cuh with the same twiddle tables (exp(-2 pi i m / L), FP32 with a
// remainder table for the compensated multiply).
#pragma once

#include "fft_block.cuh"

namespace gpe {

struct Radices {
    int n;
    int r[8];
};

// Same factorisation as the host planner (plan.hpp factor_line).
__host__ __device__ constexpr Radices radices_of(int L) {
    Radices R{0, {0, 0, 0, 0, 0, 0, 0, 0}};
    int m = L, e = 0;
    while (m % 2 == 0) {
        m /= 2;
        ++e;
    }
    if (e > 0) {
        const int st = (e + 3) / 4;
        for (int s = 0; s < st; ++s) {
            const int bits = e / st + (s < e % st ? 1 : 0);
            R.r[R.n++]     = 1 << bits;
        }
    }
    while (m % 3 == 0) {
        R.r[R.n++] = 3;
        m /= 3;
    }
    while (m % 5 == 0) {
        R.r[R.n++] = 5;
        m /= 5;
    }
    while (m % 7 == 0) {
        R.r[R.n++] = 7;
        m /= 7;
    }
    return R;
}

__host__ __device__ constexpr bool ct_supported(int L) {
    int m = L;
    for (int p : {2, 3, 5, 7})
        while (m % p == 0)
            m /= p;
    return m == 1 && radices_of(L).n <= 8;
}

template <int SIGN, class R, int L, int RADIX, int NS, int COUNT, int TS, int NT>
__device__ __forceinline__ void ct_stage(const cplx<R> *__restrict__ src, cplx<R> *__restrict__ dst,
                                         const cplx<R> *__restrict__ tw,
                                         const cplx<R> *__restrict__ twlo, int tid) {
    using C                = cplx<R>;
    constexpr int NR       = L / RADIX;
    constexpr int STEP     = L / (NS * RADIX);
    constexpr int ITEMS    = COUNT * NR;
    constexpr int ROUNDS   = (ITEMS + NT - 1) / NT;
#pragma unroll
    for (int rd = 0; rd < ROUNDS; ++rd) {
        const int it = rd * NT + tid;
        if (ITEMS % NT != 0 && it >= ITEMS)
            break;
        const int j  = it / COUNT;
        const int b  = it - j * COUNT;
        const int jm = j % NS;
        C a[RADIX];
        const C *s = src + b + j * TS;
#pragma unroll
        for (int k = 0; k < RADIX; ++k) {
            C v = s[k * NR * TS];
            if (NS > 1 && k > 0) {
                const int t = jm * k * STEP;
                const C w   = __ldg(&tw[t]);
                if constexpr (sizeof(R) == 4)
                    v = twmul<SIGN>(v, w, __ldg(&twlo[t]));
                else
                    v = SIGN < 0 ? cmul(v, w) : cmulc(v, w);
            }
            a[k] = v;
        }
        DFT<RADIX, SIGN, R>::run(a);
        const int idxD = (j / NS) * NS * RADIX + jm;
        C *d           = dst + b + idxD * TS;
#pragma unroll
        for (int q = 0; q < RADIX; ++q)
            d[q * NS * TS] = a[q];
    }
}

// Runs all stages; the tile must be complete in `src` (caller syncs before).
// Returns the buffer holding the result; syncs after every stage.
template <int SIGN, class R, int L, int COUNT, int TS, int NT, int S = 0, int NS = 1>
__device__ __forceinline__ cplx<R> *ct_fft(cplx<R> *src, cplx<R> *dst, const cplx<R> *tw,
                                           const cplx<R> *twlo, int tid) {
    constexpr Radices RAD = radices_of(L);
    if constexpr (S == RAD.n) {
        return src;
    } else {
        constexpr int RADIX = RAD.r[S];
        ct_stage<SIGN, R, L, RADIX, NS, COUNT, TS, NT>(src, dst, tw, twlo, tid);
        __syncthreads();
        return ct_fft<SIGN, R, L, COUNT, TS, NT, S + 1, NS * RADIX>(dst, src, tw, twlo, tid);
    }
}

// In-place variant: each thread first reads all the butterflies it owns in this
// stage into registers, the block synchronises, then the results are written
// back into the same buffer.  Needs one tile buffer instead of two (the
// Stockham output order is kept).  ROUNDS = ceil(COUNT*L/RADIX / NT) butterflies
// per thread are held at once.
//   CMP  compensated twiddles (needed where the norm of psi must not drift;
//        the dipolar potential's transforms run without)
//   IH   first stage: only the lower half of each line is non-zero (zero-padded
//        input); the upper half is neither read nor needs to be initialised
//   OH   last stage: only the lower half of each line is kept (cropped output)
template <int SIGN, class R, int L, int RADIX, int NS, int COUNT, int TS, int NT, bool CMP = true,
          bool IH = false, bool OH = false>
__device__ __forceinline__ void ct_stage_ip(cplx<R> *__restrict__ buf, const cplx<R> *__restrict__ tw,
                                            const cplx<R> *__restrict__ twlo, int tid) {
    using C                = cplx<R>;
    constexpr int NR       = L / RADIX;
    constexpr int STEP     = L / (NS * RADIX);
    constexpr int ITEMS    = COUNT * NR;
    constexpr int ROUNDS   = (ITEMS + NT - 1) / NT;
    C a[ROUNDS][RADIX];
#pragma unroll
    for (int rd = 0; rd < ROUNDS; ++rd) {
        const int it = rd * NT + tid;
        if (ITEMS % NT != 0 && it >= ITEMS)
            break;
        const int j  = it / COUNT;
        const int b  = it - j * COUNT;
        const int jm = j % NS;
        const C *s   = buf + b + j * TS;
#pragma unroll
        for (int k = 0; k < RADIX; ++k) {
            if (IH && NS == 1 && 2 * k >= RADIX) {
                a[rd][k] = C{(R)0, (R)0};
                continue;
            }
            C v = s[k * NR * TS];
            if (NS > 1 && k > 0) {
                const int t = jm * k * STEP;
                const C w   = __ldg(&tw[t]);
                if constexpr (sizeof(R) == 4 && CMP)
                    v = twmul<SIGN>(v, w, __ldg(&twlo[t]));
                else
                    v = SIGN < 0 ? cmul(v, w) : cmulc(v, w);
            }
            a[rd][k] = v;
        }
    }
    __syncthreads();
#pragma unroll
    for (int rd = 0; rd < ROUNDS; ++rd) {
        const int it = rd * NT + tid;
        if (ITEMS % NT != 0 && it >= ITEMS)
            break;
        const int j  = it / COUNT;
        const int b  = it - j * COUNT;
        const int jm = j % NS;
        DFT<RADIX, SIGN, R, CMP>::run(a[rd]);
        const int idxD = (j / NS) * NS * RADIX + jm;
        C *d           = buf + b + idxD * TS;
#pragma unroll
        for (int q = 0; q < RADIX; ++q)
            if (!(OH && NS * RADIX == L && 2 * q >= RADIX))
                d[q * NS * TS] = a[rd][q];
    }
    __syncthreads();
}

template <int SIGN, class R, int L, int COUNT, int TS, int NT, bool CMP = true, bool IH = false,
          bool OH = false, int S = 0, int NS = 1>
__device__ __forceinline__ void ct_fft_ip(cplx<R> *buf, const cplx<R> *tw, const cplx<R> *twlo, int tid) {
    constexpr Radices RAD = radices_of(L);
    if constexpr (S < RAD.n) {
        constexpr int RADIX = RAD.r[S];
        // pruning needs an even radix on the pruned stage
        constexpr bool ih = IH && S == 0 && RADIX % 2 == 0;
        constexpr bool oh = OH && S == RAD.n - 1 && RADIX % 2 == 0;
        ct_stage_ip<SIGN, R, L, RADIX, NS, COUNT, TS, NT, CMP, ih, oh>(buf, tw, twlo, tid);
        ct_fft_ip<SIGN, R, L, COUNT, TS, NT, CMP, IH, OH, S + 1, NS * RADIX>(buf, tw, twlo, tid);
    }
}

// Whether ct_fft_ip prunes the first / last stage of a length-L transform.
template <int L> constexpr bool ct_prunes_in() { return radices_of(L).r[0] % 2 == 0; }
template <int L> constexpr bool ct_prunes_out() {
    return radices_of(L).r[radices_of(L).n - 1] % 2 == 0;
}

// Number of stages (the result is in the first buffer when even).
template <int L> constexpr int ct_nstages() { return radices_of(L).n; }

} // namespace gpe
