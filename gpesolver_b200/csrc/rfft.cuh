// Line transforms whose first and last Stockham stages work in registers.
//
// A CTA transforms COUNT lines of length L (compile-time).  Stage 0 reads its
// butterfly inputs straight from global memory through a loader ld(b, t)
// (element t of line b) and the last stage hands its outputs to a sink
// st(b, t, v); only the stages in between go through the shared-memory tile
// (element t of line b at buf[b + t*TS]).  A two-stage transform therefore
// writes and reads the tile once, where staging the whole line through shared
// memory costs three writes and three reads.
//
// Pairing a forward and an inverse transform: the forward transform's last stage
// (radix r, Ns = L / r) leaves, in the registers of the thread that owns item j
// of line b, the outputs X[j + q L/r], q < r.  An inverse transform with the
// radices in reverse order starts with a radix-r stage whose item j reads exactly
// X[j + k L/r], k < r, and the same (j, b) -> thread mapping.  So
// run_to_regs (forward) -> pointwise multiply -> run_from_regs (inverse) needs no
// shared-memory round trip between the two transforms.
//
// Pruning (dipolar transforms of zero-padded lines): IH - the upper half of
// every input line is zero (stage 0 computes DFTZ on the lower half of its
// inputs and never loads the rest); OH - only the lower half of every output
// line is wanted (the sink is not called for the rest, and the compiler drops
// the arithmetic that only feeds them).  Both need an even radix on the pruned
// stage.
#pragma once

#include "ct_fft.cuh"

namespace gpe {

__host__ __device__ constexpr Radices reversed(Radices r) {
    Radices o{r.n, {0, 0, 0, 0, 0, 0, 0, 0}};
    for (int s = 0; s < r.n; ++s)
        o.r[s] = r.r[r.n - 1 - s];
    return o;
}

// TWS: the twiddle table passed to the stages is in shared memory (plain loads
// instead of read-only global loads).
template <int SIGN, class R, int L, int COUNT, int TS, int NT, bool CMP, bool REV, bool IH = false,
          bool OH = false, bool TWS = false>
struct LinePass {
    using C                        = cplx<R>;
    static constexpr Radices RAD   = REV ? reversed(radices_of(L)) : radices_of(L);
    static constexpr int NSTG      = RAD.n;
    static constexpr int R0        = RAD.r[0];
    static constexpr int RL        = RAD.r[NSTG - 1];
    static constexpr int NR0       = L / R0;  // stage-0 butterflies per line
    static constexpr int NSL       = L / RL;  // last-stage butterflies per line (= its Ns)
    static constexpr int ITEMS0    = COUNT * NR0;
    static constexpr int ITEMSL    = COUNT * NSL;
    static constexpr int ROUNDS0   = (ITEMS0 + NT - 1) / NT;
    static constexpr int ROUNDSL   = (ITEMSL + NT - 1) / NT;
    static_assert(!IH || R0 % 2 == 0, "input pruning needs an even first radix");
    static_assert(!OH || RL % 2 == 0, "output pruning needs an even last radix");
    static_assert(NT % COUNT == 0, "each thread keeps one line b in every round");

    static constexpr int ns_before(int S) {
        int ns = 1;
        for (int s = 0; s < S; ++s)
            ns *= RAD.r[s];
        return ns;
    }

    // item `it` of a stage with `items` butterflies: valid?
    template <int ITEMS> static __device__ __forceinline__ bool valid(int it) {
        return ITEMS % NT == 0 || it < ITEMS;
    }

    // Line index of this thread's items (the same in every round).
    static __device__ __forceinline__ int line_of(int tid) { return tid % COUNT; }
    // Element index of output q of last-stage round rd (run_to_regs layout).
    static __device__ __forceinline__ int last_index(int tid, int rd, int q) {
        return (rd * NT + tid) / COUNT + q * NSL;
    }

    static __device__ __forceinline__ void twiddle(C &v, int jm, int k, int NS, int STEP, const C *tw,
                                                   const C *twlo) {
        const int t = jm * k * STEP;
        const C w   = TWS ? tw[t] : __ldg(&tw[t]);
        if constexpr (sizeof(R) == 4 && CMP)
            v = twmul<SIGN>(v, w, TWS ? twlo[t] : __ldg(&twlo[t]));
        else
            v = SIGN < 0 ? cmul(v, w) : cmulc(v, w);
    }

    // stage 0 inputs x[j + k NR0] of line b, k < R0
    template <class Ld> static __device__ __forceinline__ void load0(C *a, Ld &ld, int j, int b) {
#pragma unroll
        for (int k = 0; k < R0; ++k) {
            if (IH && 2 * k >= R0)
                a[k] = C{(R)0, (R)0};
            else
                a[k] = ld(b, j + k * NR0);
        }
        DFTZ<R0, SIGN, R, CMP, IH ? R0 / 2 : R0>::run(a);
    }

    // Stage 0 of every round into the tile: all rounds' global loads are issued
    // before any butterfly, so a thread keeps ROUNDS0 x R0 loads in flight
    // (the lines of 512 points take four rounds).
    template <class Ld> static __device__ __forceinline__ void stage0_to_tile(C *buf, Ld &ld, int tid) {
        if constexpr (ROUNDS0 == 1) {
            if (valid<ITEMS0>(tid)) {
                const int j = tid / COUNT, b = tid - j * COUNT;
                C a[R0];
                load0(a, ld, j, b);
                store0(buf, a, j, b);
            }
        } else {
            C t[ROUNDS0][R0];
#pragma unroll
            for (int rd = 0; rd < ROUNDS0; ++rd) {
                const int it = rd * NT + tid;
                if (!valid<ITEMS0>(it))
                    break;
                const int j = it / COUNT, b = it - j * COUNT;
#pragma unroll
                for (int k = 0; k < R0; ++k)
                    t[rd][k] = (IH && 2 * k >= R0) ? C{(R)0, (R)0} : ld(b, j + k * NR0);
            }
#pragma unroll
            for (int rd = 0; rd < ROUNDS0; ++rd) {
                const int it = rd * NT + tid;
                if (!valid<ITEMS0>(it))
                    break;
                const int j = it / COUNT, b = it - j * COUNT;
                DFTZ<R0, SIGN, R, CMP, IH ? R0 / 2 : R0>::run(t[rd]);
                store0(buf, t[rd], j, b);
            }
        }
    }

    static __device__ __forceinline__ void store0(C *buf, const C *a, int j, int b) {
#pragma unroll
        for (int q = 0; q < R0; ++q)
            buf[b + (j * R0 + q) * TS] = a[q];
    }

    // last-stage inputs y[j + k NSL] (twiddled) -> a = X[j + q NSL]
    static __device__ __forceinline__ void loadL(const C *buf, C *a, int j, int b, const C *tw,
                                                 const C *twlo) {
#pragma unroll
        for (int k = 0; k < RL; ++k) {
            C v = buf[b + (j + k * NSL) * TS];
            if (k > 0)
                twiddle(v, j, k, NSL, 1, tw, twlo);
            a[k] = v;
        }
        DFT<RL, SIGN, R, CMP>::run(a);
    }

    template <int S>
    static __device__ __forceinline__ void middle(C *buf, const C *tw, const C *twlo, int tid) {
        if constexpr (S < NSTG - 1) {
            ct_stage_ip<SIGN, R, L, RAD.r[S], ns_before(S), COUNT, TS, NT, CMP, false, false>(buf, tw, twlo, tid);
            middle<S + 1>(buf, tw, twlo, tid);
        }
    }

    template <class St> static __device__ __forceinline__ void emit(St &st, const C *a, int j, int b) {
#pragma unroll
        for (int q = 0; q < RL; ++q)
            if (!(OH && 2 * q >= RL))
                st(b, j + q * NSL, a[q]);
    }

    // loader -> sink.  The tile must be free (the caller synchronises before a
    // reuse); it is in use until every thread has returned.
    template <class Ld, class St>
    static __device__ __forceinline__ void run(C *buf, Ld ld, St st, const C *tw, const C *twlo, int tid) {
        if constexpr (NSTG == 1) {
#pragma unroll
            for (int rd = 0; rd < ROUNDS0; ++rd) {
                const int it = rd * NT + tid;
                if (!valid<ITEMS0>(it))
                    break;
                C a[R0];
                load0(a, ld, 0, it);
                emit(st, a, 0, it);
            }
        } else {
            stage0_to_tile(buf, ld, tid);
            __syncthreads();
            middle<1>(buf, tw, twlo, tid);
#pragma unroll
            for (int rd = 0; rd < ROUNDSL; ++rd) {
                const int it = rd * NT + tid;
                if (!valid<ITEMSL>(it))
                    break;
                const int j = it / COUNT, b = it - j * COUNT;
                C a[RL];
                loadL(buf, a, j, b, tw, twlo);
                emit(st, a, j, b);
            }
        }
    }

    // loader -> registers: a[rd][q] = X[last_index(tid, rd, q)] of line line_of(tid).
    template <class Ld>
    static __device__ __forceinline__ void run_to_regs(C *buf, Ld ld, C (&a)[ROUNDSL][RL], const C *tw,
                                                       const C *twlo, int tid) {
        if constexpr (NSTG == 1) {
#pragma unroll
            for (int rd = 0; rd < ROUNDS0; ++rd) {
                const int it = rd * NT + tid;
                if (!valid<ITEMS0>(it))
                    break;
                load0(a[rd], ld, 0, it);
            }
        } else {
            stage0_to_tile(buf, ld, tid);
            __syncthreads();
            middle<1>(buf, tw, twlo, tid);
#pragma unroll
            for (int rd = 0; rd < ROUNDSL; ++rd) {
                const int it = rd * NT + tid;
                if (!valid<ITEMSL>(it))
                    break;
                const int j = it / COUNT, b = it - j * COUNT;
                loadL(buf, a[rd], j, b, tw, twlo);
            }
        }
    }

    // registers (the layout run_to_regs of the reversed transform leaves) -> sink.
    // The tile must be free: synchronise between run_to_regs and this call.
    template <class St>
    static __device__ __forceinline__ void run_from_regs(C *buf, C (&a)[ROUNDS0][R0], St st, const C *tw,
                                                         const C *twlo, int tid) {
        if constexpr (NSTG == 1) {
#pragma unroll
            for (int rd = 0; rd < ROUNDS0; ++rd) {
                const int it = rd * NT + tid;
                if (!valid<ITEMS0>(it))
                    break;
                DFT<R0, SIGN, R, CMP>::run(a[rd]);
                emit(st, a[rd], 0, it);
            }
        } else {
#pragma unroll
            for (int rd = 0; rd < ROUNDS0; ++rd) {
                const int it = rd * NT + tid;
                if (!valid<ITEMS0>(it))
                    break;
                const int j = it / COUNT, b = it - j * COUNT;
                DFT<R0, SIGN, R, CMP>::run(a[rd]);
                store0(buf, a[rd], j, b);
            }
            __syncthreads();
            middle<1>(buf, tw, twlo, tid);
#pragma unroll
            for (int rd = 0; rd < ROUNDSL; ++rd) {
                const int it = rd * NT + tid;
                if (!valid<ITEMSL>(it))
                    break;
                const int j = it / COUNT, b = it - j * COUNT;
                C t[RL];
                loadL(buf, t, j, b, tw, twlo);
                emit(st, t, j, b);
            }
        }
    }
};

// Block size for a pass of COUNT lines of length L: one butterfly of the
// largest radix per thread, 64..256 threads.
template <int L, int COUNT> constexpr int pass_threads() {
    int r = 1;
    for (int s = 0; s < radices_of(L).n; ++s)
        r = radices_of(L).r[s] > r ? radices_of(L).r[s] : r;
    int nt = COUNT * L / r;
    nt     = nt < 64 ? 64 : (nt > 256 ? 256 : nt);
    return (nt + 31) / 32 * 32;
}

} // namespace gpe
