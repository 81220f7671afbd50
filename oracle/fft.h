// fft.h -- test infrastructure: the FFT of the CPU oracle and of the FFTW-API
// shim the reference's PME is compiled against (FFTW3 is not installed here).
// Nothing in the product path includes this file.
//
// Complex DFT of any length, forward sign -1, unnormalised:
//   * power-of-two lengths: iterative radix-2 decimation in time (bit-reversed
//     input order, twiddles from one table of the N-th roots of unity);
//   * other lengths: recursive mixed radix (4, 2, 3, 5, then odd primes) with a
//     direct DFT inside each radix stage.
// 3-D real transforms follow FFTW's in-place r2c / c2r layout: real row (i0,i1)
// starts at ((i0*n1)+i1)*P doubles with P = 2(n2/2+1); the complex half
// spectrum (n2/2+1 per row) overwrites the buffer.  c2r is unnormalised and
// completes the half spectrum by Hermitian symmetry; it writes zeros into the
// padding doubles of each output row (FFTW leaves them unspecified).
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstddef>
#include <vector>

namespace dmd_fft {

using cd = std::complex<double>;

inline bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

struct Plan {
    int n = 0;
    std::vector<int> f;        // radix factors (mixed-radix path)
    std::vector<cd> w;         // exp(-2 pi i k / n), k < n
    std::vector<int> rev;      // bit reversal (power-of-two path)
    std::vector<cd> scratch, tmp;
};

inline void factorize(int n, std::vector<int>& f) {
    f.clear();
    for (int p : {4, 2, 3, 5}) {
        while (n % p == 0) {
            f.push_back(p);
            n /= p;
        }
    }
    for (int p = 7; n > 1; p += 2) {
        while (n % p == 0) {
            f.push_back(p);
            n /= p;
        }
    }
}

inline Plan& plan_for(int n) {
    static thread_local std::vector<Plan> plans;
    for (auto& p : plans)
        if (p.n == n) return p;
    Plan p;
    p.n = n;
    p.w.resize(n);
    const double pi = 3.14159265358979323846;
    for (int k = 0; k < n; ++k) {
        const double a = -2.0 * pi * static_cast<double>(k) / n;
        p.w[k] = cd(std::cos(a), std::sin(a));
    }
    if (is_pow2(n)) {
        int bits = 0;
        while ((1 << bits) < n) ++bits;
        p.rev.resize(n);
        for (int i = 0; i < n; ++i) {
            int r = 0;
            for (int b = 0; b < bits; ++b)
                if (i & (1 << b)) r |= 1 << (bits - 1 - b);
            p.rev[i] = r;
        }
    } else {
        factorize(n, p.f);
    }
    p.scratch.resize(n);
    p.tmp.resize(n);
    plans.push_back(std::move(p));
    return plans.back();
}

// Decimation in time: X[k + q m] = sum_r W_n^{r(k+qm)} Y_r[k], Y_r = DFT_m(x[r::p]).
inline void fft_rec(const cd* in, int is, cd* out, int n, int level, Plan& P, bool inv) {
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    const int p = P.f[level], m = n / p;
    for (int r = 0; r < p; ++r) fft_rec(in + r * is, is * p, out + r * m, m, level + 1, P, inv);
    const int N = P.n, step = N / n;
    cd* res = P.scratch.data();
    std::vector<cd> tt(p);
    for (int k = 0; k < m; ++k) {
        for (int r = 0; r < p; ++r) {
            cd wv = P.w[(static_cast<long>(r) * k % n) * step];
            if (inv) wv = std::conj(wv);
            tt[r] = out[r * m + k] * wv;
        }
        for (int q = 0; q < p; ++q) {
            cd acc = 0;
            for (int r = 0; r < p; ++r) {
                cd wv = P.w[(static_cast<long>(r) * q % p) * (N / p)];
                if (inv) wv = std::conj(wv);
                acc += tt[r] * wv;
            }
            res[k + q * m] = acc;
        }
    }
    std::copy(res, res + n, out);
}

// In-place length-n transform; sign -1 forward, +1 backward (unnormalised).
inline void fft1d(cd* a, int n, int sign) {
    Plan& P = plan_for(n);
    const bool inv = sign > 0;
    if (!P.rev.empty()) {
        for (int i = 0; i < n; ++i)
            if (i < P.rev[i]) std::swap(a[i], a[P.rev[i]]);
        for (int len = 2; len <= n; len <<= 1) {
            const int half = len >> 1, stride = n / len;
            for (int s = 0; s < n; s += len)
                for (int k = 0; k < half; ++k) {
                    cd wv = P.w[k * stride];
                    if (inv) wv = std::conj(wv);
                    const cd t = a[s + k + half] * wv;
                    a[s + k + half] = a[s + k] - t;
                    a[s + k] += t;
                }
        }
        return;
    }
    std::copy(a, a + n, P.tmp.begin());
    fft_rec(P.tmp.data(), 1, a, n, 0, P, inv);
}

// 3-D complex transform in place over an n0*n1*n2 array, index (i0*n1 + i1)*n2 + i2.
inline void fft3d(std::vector<cd>& a, int n0, int n1, int n2, int sign) {
    const size_t s1 = static_cast<size_t>(n2), s0 = static_cast<size_t>(n1) * n2;
    for (int i0 = 0; i0 < n0; ++i0)
        for (int i1 = 0; i1 < n1; ++i1) fft1d(&a[i0 * s0 + i1 * s1], n2, sign);
    std::vector<cd> line(std::max(n0, n1));
    for (int i0 = 0; i0 < n0; ++i0)
        for (int i2 = 0; i2 < n2; ++i2) {
            for (int i1 = 0; i1 < n1; ++i1) line[i1] = a[i0 * s0 + i1 * s1 + i2];
            fft1d(line.data(), n1, sign);
            for (int i1 = 0; i1 < n1; ++i1) a[i0 * s0 + i1 * s1 + i2] = line[i1];
        }
    for (int i1 = 0; i1 < n1; ++i1)
        for (int i2 = 0; i2 < n2; ++i2) {
            for (int i0 = 0; i0 < n0; ++i0) line[i0] = a[i0 * s0 + i1 * s1 + i2];
            fft1d(line.data(), n0, sign);
            for (int i0 = 0; i0 < n0; ++i0) a[i0 * s0 + i1 * s1 + i2] = line[i0];
        }
}

// FFTW-style r2c of a real array (row pitch `pitch` doubles, n2 used) into the
// half spectrum written at `out` (n2/2+1 complex per row, interleaved doubles).
// `in` and `out` may be the same buffer (in-place, pitch = 2(n2/2+1)).
inline void r2c3d(const double* in, size_t pitch, double* out, int n0, int n1, int n2) {
    const int H = n2 / 2 + 1;
    std::vector<cd> a(static_cast<size_t>(n0) * n1 * n2);
    for (size_t row = 0; row < static_cast<size_t>(n0) * n1; ++row)
        for (int x = 0; x < n2; ++x) a[row * n2 + x] = in[row * pitch + x];
    fft3d(a, n0, n1, n2, -1);
    for (size_t row = 0; row < static_cast<size_t>(n0) * n1; ++row)
        for (int k = 0; k < H; ++k) {
            const cd v = a[row * n2 + k];
            out[(row * H + k) * 2] = v.real();
            out[(row * H + k) * 2 + 1] = v.imag();
        }
}

// Unnormalised c2r from the half spectrum `in` into real rows of pitch `pitch`
// (padding doubles zeroed); in == out allowed (in-place).
inline void c2r3d(const double* in, double* out, size_t pitch, int n0, int n1, int n2) {
    const int H = n2 / 2 + 1;
    std::vector<cd> a(static_cast<size_t>(n0) * n1 * n2);
    for (int i0 = 0; i0 < n0; ++i0)
        for (int i1 = 0; i1 < n1; ++i1)
            for (int k = 0; k < n2; ++k) {
                cd v;
                if (k < H) {
                    const size_t o = ((static_cast<size_t>(i0) * n1 + i1) * H + k) * 2;
                    v = cd(in[o], in[o + 1]);
                } else {
                    const int j0 = (n0 - i0) % n0, j1 = (n1 - i1) % n1, kk = n2 - k;
                    const size_t o = ((static_cast<size_t>(j0) * n1 + j1) * H + kk) * 2;
                    v = std::conj(cd(in[o], in[o + 1]));
                }
                a[(static_cast<size_t>(i0) * n1 + i1) * n2 + k] = v;
            }
    fft3d(a, n0, n1, n2, +1);
    for (size_t row = 0; row < static_cast<size_t>(n0) * n1; ++row) {
        for (int x = 0; x < n2; ++x) out[row * pitch + x] = a[row * n2 + x].real();
        for (size_t x = n2; x < pitch; ++x) out[row * pitch + x] = 0.0;
    }
}

}  // namespace dmd_fft
