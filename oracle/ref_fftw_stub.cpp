/* Discrete Fourier transforms behind oracle/stubs/fftw3.h -- TEST
 * INFRASTRUCTURE, linked only into oracle/_ref/scrimppp_ref_orig so that the
 * reference's PreSCRIMP (scrimppp/src/ScrimpppOrig.cpp) runs unchanged.
 *
 *   out[k] = sum_j in[j] * exp(sign * 2 pi i * j * k / n),  unnormalised.
 *
 * Power-of-two n: iterative radix-2 Cooley-Tukey (decimation in time, input
 * in bit-reversed order).  Other n: the direct O(n^2) sum, with j*k reduced
 * modulo n so that every twiddle comes from the table.  The twiddle table is
 * built once per plan from cos/sin of 2 pi t / n (no recurrence), so
 * each transform's error is a few ulps times log2(n) (radix 2) or sqrt(n)
 * (direct) of the input's norm, the same order as FFTW's.  Out-of-place
 * only, which is all the reference asks for. */
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "stubs/fftw3.h"

struct oracle_fft_plan {
    int n;
    int sign;
    fftw_complex* in;
    fftw_complex* out;
    std::vector<double> wr, wi;  // exp(sign * 2 pi i t / n), t < n
};

extern "C" {

void* fftw_malloc(size_t n) {
    void* p = nullptr;
    if (posix_memalign(&p, 64, n ? n : 1) != 0) return nullptr;
    return p;
}

void fftw_free(void* p) { std::free(p); }

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned) {
    if (n <= 0) return nullptr;
    oracle_fft_plan* p = new oracle_fft_plan;
    p->n = n;
    p->sign = sign < 0 ? -1 : 1;
    p->in = in;
    p->out = out;
    p->wr.resize(n);
    p->wi.resize(n);
    const double two_pi = 6.283185307179586476925286766559;
    for (int t = 0; t < n; ++t) {
        const double a = two_pi * (double)t / (double)n;
        p->wr[t] = std::cos(a);
        p->wi[t] = p->sign * std::sin(a);
    }
    return p;
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

static void dft_direct(const oracle_fft_plan& p) {
    const int n = p.n;
    std::vector<double> re(n), im(n);
    for (int k = 0; k < n; ++k) {
        double sr = 0.0, si = 0.0;
        int64_t t = 0;  // j * k mod n
        for (int j = 0; j < n; ++j) {
            const double xr = p.in[j][0], xi = p.in[j][1];
            sr += xr * p.wr[t] - xi * p.wi[t];
            si += xr * p.wi[t] + xi * p.wr[t];
            t += k;
            if (t >= n) t -= n;
        }
        re[k] = sr;
        im[k] = si;
    }
    for (int k = 0; k < n; ++k) {
        p.out[k][0] = re[k];
        p.out[k][1] = im[k];
    }
}

static void fft_radix2(const oracle_fft_plan& p) {
    const int n = p.n;
    int bits = 0;
    while ((1 << bits) < n) ++bits;
    std::vector<double> re(n), im(n);
    for (int j = 0; j < n; ++j) {
        int r = 0;
        for (int b = 0; b < bits; ++b) r |= ((j >> b) & 1) << (bits - 1 - b);
        re[r] = p.in[j][0];
        im[r] = p.in[j][1];
    }
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1, stride = n / len;
        for (int s = 0; s < n; s += len) {
            for (int k = 0; k < half; ++k) {
                const double cr = p.wr[k * stride], ci = p.wi[k * stride];
                const int a = s + k, b = s + k + half;
                const double tr = re[b] * cr - im[b] * ci;
                const double ti = re[b] * ci + im[b] * cr;
                re[b] = re[a] - tr;
                im[b] = im[a] - ti;
                re[a] += tr;
                im[a] += ti;
            }
        }
    }
    for (int k = 0; k < n; ++k) {
        p.out[k][0] = re[k];
        p.out[k][1] = im[k];
    }
}

void fftw_execute(const fftw_plan p) {
    if (!p) return;
    if ((p->n & (p->n - 1)) == 0) fft_radix2(*p);
    else dft_direct(*p);
}

}  // extern "C"
