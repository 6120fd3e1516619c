// Host-side FFT planning and FP64 table construction.
#pragma once

#include "fft_block.cuh"

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

namespace gpe {

// Message of the last failed gpe_* call on the calling thread (gpe_last_error).
std::string &last_error();

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// Radices of a length-L line: the power-of-two part in as few balanced stages of
// radix <= 16 as possible, then one stage per factor 3, 5 or 7.  Lengths with a
// prime factor above 7 are rejected (GPE_ERR_SIZE).
inline std::vector<int> factor_line(int L) {
    if (L < 1)
        throw Error(2, "FFT length must be positive, got " + std::to_string(L));
    std::vector<int> r;
    int m = L, e = 0;
    while (m % 2 == 0) {
        m /= 2;
        ++e;
    }
    if (e > 0) {
        const int stages = (e + 3) / 4;
        for (int s = 0; s < stages; ++s) {
            const int bits = e / stages + (s < e % stages ? 1 : 0);
            r.push_back(1 << bits);
        }
    }
    for (int p : {3, 5, 7})
        while (m % p == 0) {
            r.push_back(p);
            m /= p;
        }
    if (m != 1)
        throw Error(2, "FFT length " + std::to_string(L) +
                           " has a prime factor above 7; supported grid sizes factor into 2, 3, 5, 7");
    if (r.size() > 8)
        throw Error(2, "FFT length " + std::to_string(L) + " needs more than 8 stages");
    return r;
}

// exp(-2 pi i m / L), m < L, in FP64 (angle reduced by octant symmetry is not
// needed: cos/sin of 2 pi m / L are correctly rounded to ~1 ulp by libm).
inline std::vector<double> twiddles(int L) {
    std::vector<double> t(2 * (size_t)L);
    for (int m = 0; m < L; ++m) {
        const double a = 2.0 * M_PI * (double)m / (double)L;
        t[2 * m]       = std::cos(a);
        t[2 * m + 1]   = -std::sin(a);
    }
    return t;
}

} // namespace gpe
