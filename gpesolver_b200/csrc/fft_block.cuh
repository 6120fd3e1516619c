// Block-level FFT building blocks for sm_100a.
//
// A CTA transforms a tile of `count` independent lines of length L held in
// shared memory: element t of line b sits at s[b*bs + t*ts].  Each stage of the
// mixed-radix Stockham auto-sort algorithm (radix r in {2,3,4,5,7,8,16}) maps
// one thread to one r-point butterfly held in registers:
//
//   a_k = src[j + k L/r] * W_{Ns r}^{(j mod Ns) k}            k < r
//   b   = DFT_r(a)                                            (in registers)
//   dst[(j / Ns) Ns r + (j mod Ns) + q Ns] = b_q               q < r
//
// ping-ponging between two shared-memory buffers, so the output is in natural
// order without a bit-reversal pass.  Twiddles come from a per-length table
// exp(-2 pi i m / L), m < L, computed in FP64 and rounded once to the working
// precision (in FP32 with a second table holding the rounding remainder, for a
// compensated multiply); the inverse transform uses the conjugate.
#pragma once

#include <cuda_runtime.h>

namespace gpe {

template <class R> struct cvec;
template <> struct cvec<float> { using T = float2; };
template <> struct cvec<double> { using T = double2; };
template <class R> using cplx = typename cvec<R>::T;

template <class C> __device__ __forceinline__ C cadd(C a, C b) { return C{a.x + b.x, a.y + b.y}; }
template <class C> __device__ __forceinline__ C csub(C a, C b) { return C{a.x - b.x, a.y - b.y}; }
// complex64 sums as one packed FP32x2 instruction (sm_100 add.rn.f32x2; the
// negation folds into the operand): per component the same IEEE
// round-to-nearest result as the scalar pair, in half the issue slots
// (radix-16 DFT: 24-30% fewer instructions)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __fadd2_rn(a, float2{-b.x, -b.y}); }
template <class C> __device__ __forceinline__ C cmul(C a, C b) {
    return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a * conj(b)
template <class C> __device__ __forceinline__ C cmulc(C a, C b) {
    return C{a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <class C, class R> __device__ __forceinline__ C cscale(C a, R s) { return C{a.x * s, a.y * s}; }
// a * (SIGN * i)
template <int SIGN, class C> __device__ __forceinline__ C mul_si(C a) {
    return SIGN > 0 ? C{-a.y, a.x} : C{a.y, -a.x};
}
// a * W where W = cos + SIGN*i*sin
template <int SIGN, class C, class R> __device__ __forceinline__ C mul_w(C a, R c, R s) {
    return SIGN > 0 ? C{a.x * c - a.y * s, a.x * s + a.y * c} : C{a.x * c + a.y * s, a.y * c - a.x * s};
}

// Twiddles are applied with a compensated multiply in FP32: each twiddle is
// split as hi + lo (hi = the float nearest the exact value, lo = the float
// nearest the remainder) and x*c is evaluated as fma(x, hi, x*lo), which rounds
// once to the correctly rounded x*c.  A plain FP32 twiddle carries a fixed
// modulus error (2 fl32(sqrt(1/2))^2 - 1 = -3.4e-8, c8^2 + s8^2 - 1 = -5.7e-8,
// and a net negative mean over a twiddle table) that every butterfly applies
// with the same sign, so the norm of psi drifted by ~5e-8 per FFT round trip;
// compensated, the drift is at the 1e-11 noise level.
template <class R> __device__ __forceinline__ R cmulk(R x, double c) {
    if constexpr (sizeof(R) == 4) {
        const float hi = (float)c;
        const float lo = (float)(c - (double)hi);
        return fmaf(x, hi, x * lo);
    } else {
        return x * c;
    }
}
// a * W where W = c + SIGN*i*s, compensated
template <int SIGN, class C, class R> __device__ __forceinline__ C mul_wk(C a, double c, double s) {
    if (SIGN > 0)
        return C{cmulk<R>(a.x, c) - cmulk<R>(a.y, s), cmulk<R>(a.x, s) + cmulk<R>(a.y, c)};
    return C{cmulk<R>(a.x, c) + cmulk<R>(a.y, s), cmulk<R>(a.y, c) - cmulk<R>(a.x, s)};
}

// cos / sin of 2 pi m / 16 (the twiddles of the radix-8 and radix-16 kernels)
__device__ __forceinline__ double cos16(int m) {
    constexpr double c8 = 0.92387953251128675613, s8 = 0.38268343236508977173,
                     r2 = 0.70710678118654752440;
    switch (m & 15) {
    case 0: return 1.0;
    case 1: return c8;
    case 2: return r2;
    case 3: return s8;
    case 4: return 0.0;
    case 5: return -s8;
    case 6: return -r2;
    case 7: return -c8;
    case 8: return -1.0;
    case 9: return -c8;
    case 10: return -r2;
    case 11: return -s8;
    case 12: return 0.0;
    case 13: return s8;
    case 14: return r2;
    default: return c8;
    }
}
__device__ __forceinline__ double sin16(int m) { return cos16(m - 4); }

// CMP: apply the radix-8/16/3/5/7 constants with the compensated multiply.
template <int N, int SIGN, class R, bool CMP = true> struct DFT;

template <int SIGN, class C, class R, bool CMP> __device__ __forceinline__ C mul_wc(C a, double c, double s) {
    if constexpr (CMP)
        return mul_wk<SIGN, C, R>(a, c, s);
    else
        return mul_w<SIGN>(a, (R)c, (R)s);
}

template <int SIGN, class R, bool CMP> struct DFT<2, SIGN, R, CMP> {
    using C = cplx<R>;
    static __device__ __forceinline__ void run(C *a) {
        C t = a[0];
        a[0] = cadd(t, a[1]);
        a[1] = csub(t, a[1]);
    }
};

template <int SIGN, class R, bool CMP> struct DFT<4, SIGN, R, CMP> {
    using C = cplx<R>;
    static __device__ __forceinline__ void run(C *a) {
        C t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]);
        C t2 = cadd(a[1], a[3]), d = csub(a[1], a[3]);
        a[0] = cadd(t0, t2);
        a[2] = csub(t0, t2);
        // t1 +- SIGN i d, component by component (a packed form would first
        // have to assemble the swapped pair)
        if (SIGN > 0) {
            a[1] = C{t1.x - d.y, t1.y + d.x};
            a[3] = C{t1.x + d.y, t1.y - d.x};
        } else {
            a[1] = C{t1.x + d.y, t1.y - d.x};
            a[3] = C{t1.x - d.y, t1.y + d.x};
        }
    }
};

// N = N1 * N2 split in registers: x[N2 n1 + n2] -> X[k1 + N1 k2]
//   y[n2][k1] = DFT_N1(x[N2 n1 + n2]) * W_N^{n2 k1};  X[k1 + N1 k2] = DFT_N2(y[.][k1])
//   Z1 < N1: only x[N2 n1 + n2] with n1 < Z1 are non-zero (the first N Z1 / N1
//   inputs); the zeros are neither read nor added (DFTZ below).
template <int N, int SIGN, class R, bool CMP, int ZIN> struct DFTZ;
template <int N1, int N2, int SIGN, class R, bool CMP = true, int Z1 = N1> struct DFTSplit {
    using C = cplx<R>;
    static __device__ __forceinline__ void run(C *a) {
        constexpr int N = N1 * N2;
        C y[N2][N1];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) {
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1)
                y[n2][n1] = n1 < Z1 ? a[N2 * n1 + n2] : C{(R)0, (R)0};
            DFTZ<N1, SIGN, R, CMP, Z1>::run(y[n2]);
#pragma unroll
            for (int k1 = 0; k1 < N1; ++k1) {
                const int m = (n2 * k1 * (16 / N)) & 15;
                if (m == 4 || m == 12)
                    y[n2][k1] = (m == 4) == (SIGN > 0) ? mul_si<+1>(y[n2][k1]) : mul_si<-1>(y[n2][k1]);
                else if (m == 8)
                    y[n2][k1] = C{-y[n2][k1].x, -y[n2][k1].y};
                else if (m != 0)
                    y[n2][k1] = mul_wc<SIGN, C, R, CMP>(y[n2][k1], cos16(m), sin16(m));
            }
        }
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) {
            C z[N2];
#pragma unroll
            for (int n2 = 0; n2 < N2; ++n2)
                z[n2] = y[n2][k1];
            DFT<N2, SIGN, R, CMP>::run(z);
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2)
                a[k1 + N1 * k2] = z[k2];
        }
    }
};

template <int SIGN, class R, bool CMP> struct DFT<8, SIGN, R, CMP> {
    static __device__ __forceinline__ void run(cplx<R> *a) { DFTSplit<4, 2, SIGN, R, CMP>::run(a); }
};
template <int SIGN, class R, bool CMP> struct DFT<16, SIGN, R, CMP> {
    static __device__ __forceinline__ void run(cplx<R> *a) { DFTSplit<4, 4, SIGN, R, CMP>::run(a); }
};

// DFT of N points of which only the first ZIN are non-zero (ZIN = N or N / 2):
// the pruned first stage of a zero-padded transform.  a[ZIN..N-1] are not read.
template <int N, int SIGN, class R, bool CMP, int ZIN> struct DFTZ {
    static_assert(ZIN == N, "pruned DFT: N in {2, 4, 8, 16} with ZIN = N / 2");
    static __device__ __forceinline__ void run(cplx<R> *a) { DFT<N, SIGN, R, CMP>::run(a); }
};
template <int SIGN, class R, bool CMP> struct DFTZ<2, SIGN, R, CMP, 1> {
    static __device__ __forceinline__ void run(cplx<R> *a) { a[1] = a[0]; }
};
template <int SIGN, class R, bool CMP> struct DFTZ<4, SIGN, R, CMP, 2> {
    using C = cplx<R>;
    static __device__ __forceinline__ void run(C *a) {
        const C x0 = a[0], x1 = a[1];
        a[0] = cadd(x0, x1);
        a[2] = csub(x0, x1);
        if (SIGN > 0) { // x0 +- SIGN i x1
            a[1] = C{x0.x - x1.y, x0.y + x1.x};
            a[3] = C{x0.x + x1.y, x0.y - x1.x};
        } else {
            a[1] = C{x0.x + x1.y, x0.y - x1.x};
            a[3] = C{x0.x - x1.y, x0.y + x1.x};
        }
    }
};
template <int SIGN, class R, bool CMP> struct DFTZ<8, SIGN, R, CMP, 4> {
    static __device__ __forceinline__ void run(cplx<R> *a) { DFTSplit<4, 2, SIGN, R, CMP, 2>::run(a); }
};
template <int SIGN, class R, bool CMP> struct DFTZ<16, SIGN, R, CMP, 8> {
    static __device__ __forceinline__ void run(cplx<R> *a) { DFTSplit<4, 4, SIGN, R, CMP, 2>::run(a); }
};

// Odd prime radices: direct r-point sums with the constant table cos/sin(2 pi m / r).
template <int P> struct OddTab;
template <> struct OddTab<3> {
    static __device__ __forceinline__ double c(int m) { return m == 0 ? 1.0 : -0.5; }
    static __device__ __forceinline__ double s(int m) {
        return m == 0 ? 0.0 : (m == 1 ? 0.86602540378443864676 : -0.86602540378443864676);
    }
};
template <> struct OddTab<5> {
    static __device__ __forceinline__ double c(int m) {
        constexpr double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
        return m == 0 ? 1.0 : (m == 1 || m == 4) ? c1 : c2;
    }
    static __device__ __forceinline__ double s(int m) {
        constexpr double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
        switch (m) {
        case 1: return s1;
        case 2: return s2;
        case 3: return -s2;
        case 4: return -s1;
        default: return 0.0;
        }
    }
};
template <> struct OddTab<7> {
    static __device__ __forceinline__ double c(int m) {
        constexpr double c1 = 0.62348980185873353053, c2 = -0.22252093395631440429,
                         c3 = -0.90096886790241912624;
        switch (m) {
        case 0: return 1.0;
        case 1: case 6: return c1;
        case 2: case 5: return c2;
        default: return c3;
        }
    }
    static __device__ __forceinline__ double s(int m) {
        constexpr double s1 = 0.78183148246802980871, s2 = 0.97492791218182360702,
                         s3 = 0.43388373911755812048;
        switch (m) {
        case 1: return s1;
        case 2: return s2;
        case 3: return s3;
        case 4: return -s3;
        case 5: return -s2;
        case 6: return -s1;
        default: return 0.0;
        }
    }
};

template <int P, int SIGN, class R, bool CMP = true> struct DFTOdd {
    using C = cplx<R>;
    static __device__ __forceinline__ void run(C *a) {
        C out[P];
#pragma unroll
        for (int q = 0; q < P; ++q) {
            C acc = a[0];
#pragma unroll
            for (int k = 1; k < P; ++k) {
                const int m = (k * q) % P;
                acc         = cadd(acc, mul_wc<SIGN, C, R, CMP>(a[k], OddTab<P>::c(m), OddTab<P>::s(m)));
            }
            out[q] = acc;
        }
#pragma unroll
        for (int q = 0; q < P; ++q)
            a[q] = out[q];
    }
};
template <int SIGN, class R, bool CMP> struct DFT<3, SIGN, R, CMP> {
    static __device__ __forceinline__ void run(cplx<R> *a) { DFTOdd<3, SIGN, R, CMP>::run(a); }
};
template <int SIGN, class R, bool CMP> struct DFT<5, SIGN, R, CMP> {
    static __device__ __forceinline__ void run(cplx<R> *a) { DFTOdd<5, SIGN, R, CMP>::run(a); }
};
template <int SIGN, class R, bool CMP> struct DFT<7, SIGN, R, CMP> {
    static __device__ __forceinline__ void run(cplx<R> *a) { DFTOdd<7, SIGN, R, CMP>::run(a); }
};

// Plan of one line transform of length L (host-built; passed by value).
struct LinePlan {
    int L;
    int nstages;
    int radix[8];
    const void *tw;   // cplx<R>[L]: exp(-2 pi i m / L), rounded to R
    const void *twlo; // FP32 only: cplx<R>[L], the rounding remainder of tw
};

// v * w (SIGN < 0) or v * conj(w) (SIGN > 0) with w = hi + lo (compensated).
template <int SIGN, class C> __device__ __forceinline__ C twmul(C v, C hi, C lo) {
    const float sh = SIGN < 0 ? hi.y : -hi.y, sl = SIGN < 0 ? lo.y : -lo.y;
    const float cre = v.x * lo.x - v.y * sl;
    const float cim = v.x * sl + v.y * lo.x;
    return C{fmaf(v.x, hi.x, fmaf(-v.y, sh, cre)), fmaf(v.x, sh, fmaf(v.y, hi.x, cim))};
}

template <int RADIX, int SIGN, class R>
__device__ __forceinline__ void fft_stage(const cplx<R> *__restrict__ src, cplx<R> *__restrict__ dst,
                                          int L, int Ns, int count, int bs, int ts,
                                          const cplx<R> *__restrict__ tw,
                                          const cplx<R> *__restrict__ twlo, int tid, int nthreads) {
    using C         = cplx<R>;
    const int nr    = L / RADIX;
    const int step  = L / (Ns * RADIX);
    const int items = count * nr;
    // consecutive threads take consecutive lines b: with the tile layouts used
    // here (bs = 1) their shared-memory accesses fall in distinct banks.
    for (int it = tid; it < items; it += nthreads) {
        const int j  = it / count;
        const int b  = it - j * count;
        const int jm = j % Ns;
        C a[RADIX];
        const C *s = src + (size_t)b * bs + (size_t)j * ts;
#pragma unroll
        for (int k = 0; k < RADIX; ++k) {
            C v = s[(size_t)k * nr * ts];
            if (k > 0 && jm > 0) {
                const int t = jm * k * step; // < Ns * RADIX * step = L
                const C w   = __ldg(&tw[t]);
                if constexpr (sizeof(R) == 4)
                    v = twmul<SIGN>(v, w, __ldg(&twlo[t]));
                else
                    v = SIGN < 0 ? cmul(v, w) : cmulc(v, w);
            }
            a[k] = v;
        }
        DFT<RADIX, SIGN, R>::run(a);
        const int idxD = (j / Ns) * Ns * RADIX + jm;
        C *d           = dst + (size_t)b * bs + (size_t)idxD * ts;
#pragma unroll
        for (int q = 0; q < RADIX; ++q)
            d[(size_t)q * Ns * ts] = a[q];
    }
}

// Transforms the tile in buf0 (using buf1 as the second Stockham buffer).
// Requires the tile to be complete in shared memory (caller syncs before);
// syncs after every stage.  Returns the buffer that holds the result.
template <int SIGN, class R>
__device__ cplx<R> *block_fft(cplx<R> *buf0, cplx<R> *buf1, const LinePlan &ln, int count, int bs,
                              int ts, int tid, int nthreads) {
    using C     = cplx<R>;
    C *src      = buf0;
    C *dst      = buf1;
    int Ns      = 1;
    const C *tw = reinterpret_cast<const C *>(ln.tw);
    const C *tl = reinterpret_cast<const C *>(ln.twlo);
    for (int s = 0; s < ln.nstages; ++s) {
        const int r = ln.radix[s];
        switch (r) {
        case 2: fft_stage<2, SIGN, R>(src, dst, ln.L, Ns, count, bs, ts, tw, tl, tid, nthreads); break;
        case 3: fft_stage<3, SIGN, R>(src, dst, ln.L, Ns, count, bs, ts, tw, tl, tid, nthreads); break;
        case 4: fft_stage<4, SIGN, R>(src, dst, ln.L, Ns, count, bs, ts, tw, tl, tid, nthreads); break;
        case 5: fft_stage<5, SIGN, R>(src, dst, ln.L, Ns, count, bs, ts, tw, tl, tid, nthreads); break;
        case 7: fft_stage<7, SIGN, R>(src, dst, ln.L, Ns, count, bs, ts, tw, tl, tid, nthreads); break;
        case 8: fft_stage<8, SIGN, R>(src, dst, ln.L, Ns, count, bs, ts, tw, tl, tid, nthreads); break;
        default: fft_stage<16, SIGN, R>(src, dst, ln.L, Ns, count, bs, ts, tw, tl, tid, nthreads); break;
        }
        __syncthreads();
        C *t = src;
        src  = dst;
        dst  = t;
        Ns *= r;
    }
    return src;
}

} // namespace gpe
