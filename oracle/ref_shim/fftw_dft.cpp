/*
 * The transforms declared in ref_shim/fftw3.h: FFTW 3's documented complex and
 * real-data DFTs, evaluated as direct sums per line (see the header for the
 * definition restated).  Test infrastructure only; linked into the oracle
 * libraries built from the reference's sources, never into the product.
 */
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

using cld = std::complex<long double>;
constexpr int MAXR = 8;
const long double TWO_PI = 6.283185307179586476925286766559005768L;

enum Kind { C2C = 0, R2C = 1, C2R = 2 };

}  // namespace

struct qsref_fftw_plan_s {
    Kind kind;
    int rank;
    int n[MAXR];
    int howmany;
    int inembed[MAXR], onembed[MAXR];
    int istride, idist, ostride, odist;
    int sign;
    void* in;
    void* out;
};

namespace {

long long product(const int* n, int r) {
    long long p = 1;
    for (int d = 0; d < r; ++d) p *= n[d];
    return p;
}

// row-major linear index of multi-index `idx` in an array of dimensions `dims`
long long rowmajor(const int* idx, const int* dims, int r) {
    long long li = 0;
    for (int d = 0; d < r; ++d) li = li * dims[d] + idx[d];
    return li;
}

void unravel(long long li, const int* n, int r, int* idx) {
    for (int d = r - 1; d >= 0; --d) {
        idx[d] = (int)(li % n[d]);
        li /= n[d];
    }
}

// in-place separable DFT of a contiguous row-major block of dimensions n
void dft_block(std::vector<cld>& a, const int* n, int r, int sign) {
    const long long total = product(n, r);
    for (int d = 0; d < r; ++d) {
        const int nd = n[d];
        if (nd == 1) continue;
        std::vector<cld> w(nd), line(nd), res(nd);
        for (int m = 0; m < nd; ++m) {
            const long double ang = TWO_PI * (long double)m / (long double)nd;
            w[m] = cld(cosl(ang), (long double)sign * sinl(ang));
        }
        long long inner = 1;
        for (int e = d + 1; e < r; ++e) inner *= n[e];
        const long long outer = total / (inner * nd);
        for (long long o = 0; o < outer; ++o) {
            for (long long i = 0; i < inner; ++i) {
                const long long base = o * inner * nd + i;
                for (int j = 0; j < nd; ++j) line[j] = a[base + (long long)j * inner];
                for (int k = 0; k < nd; ++k) {
                    cld s = 0;
                    for (int j = 0; j < nd; ++j) s += line[j] * w[(int)(((long long)j * k) % nd)];
                    res[k] = s;
                }
                for (int k = 0; k < nd; ++k) a[base + (long long)k * inner] = res[k];
            }
        }
    }
}

fftw_plan make_plan(Kind kind, int rank, const int* n, int howmany, void* in, const int* inembed, int istride,
                    int idist, void* out, const int* onembed, int ostride, int odist, int sign) {
    if (rank < 1 || rank > MAXR || howmany < 0) return nullptr;
    fftw_plan p = new qsref_fftw_plan_s();
    p->kind = kind;
    p->rank = rank;
    p->howmany = howmany;
    for (int d = 0; d < rank; ++d) {
        if (n[d] < 1) {
            delete p;
            return nullptr;
        }
        p->n[d] = n[d];
        p->inembed[d] = inembed ? inembed[d] : n[d];
        p->onembed[d] = onembed ? onembed[d] : n[d];
    }
    p->istride = istride;
    p->idist = idist;
    p->ostride = ostride;
    p->odist = odist;
    p->sign = sign;
    p->in = in;
    p->out = out;
    return p;
}

void exec_c2c(const qsref_fftw_plan_s* p, fftw_complex* in, fftw_complex* out) {
    const int r = p->rank;
    const long long total = product(p->n, r);
    std::vector<cld> a((size_t)total);
    int idx[MAXR];
    for (int b = 0; b < p->howmany; ++b) {
        const fftw_complex* src = in + (long long)b * p->idist;
        for (long long li = 0; li < total; ++li) {
            unravel(li, p->n, r, idx);
            const long long off = (long long)p->istride * rowmajor(idx, p->inembed, r);
            a[(size_t)li] = cld(src[off][0], src[off][1]);
        }
        dft_block(a, p->n, r, p->sign);
        fftw_complex* dst = out + (long long)b * p->odist;
        for (long long li = 0; li < total; ++li) {
            unravel(li, p->n, r, idx);
            const long long off = (long long)p->ostride * rowmajor(idx, p->onembed, r);
            dst[off][0] = (double)a[(size_t)li].real();
            dst[off][1] = (double)a[(size_t)li].imag();
        }
    }
}

// contiguous real <-> half-spectrum (last dimension n/2 + 1) transforms
void exec_r2c(const qsref_fftw_plan_s* p, const double* in, fftw_complex* out) {
    const int r = p->rank;
    const long long total = product(p->n, r);
    const int nl = p->n[r - 1], nh = nl / 2 + 1;
    std::vector<cld> a((size_t)total);
    for (long long li = 0; li < total; ++li) a[(size_t)li] = cld(in[li], 0.0L);
    dft_block(a, p->n, r, FFTW_FORWARD);
    const long long rows = total / nl;
    for (long long row = 0; row < rows; ++row)
        for (int k = 0; k < nh; ++k) {
            out[row * nh + k][0] = (double)a[(size_t)(row * nl + k)].real();
            out[row * nh + k][1] = (double)a[(size_t)(row * nl + k)].imag();
        }
}

void exec_c2r(const qsref_fftw_plan_s* p, const fftw_complex* in, double* out) {
    const int r = p->rank;
    const long long total = product(p->n, r);
    const int nl = p->n[r - 1], nh = nl / 2 + 1;
    std::vector<cld> a((size_t)total);
    int idx[MAXR], neg[MAXR], hdims[MAXR];
    for (int d = 0; d < r; ++d) hdims[d] = p->n[d];
    hdims[r - 1] = nh;
    for (long long li = 0; li < total; ++li) {
        unravel(li, p->n, r, idx);
        if (idx[r - 1] < nh) {
            const fftw_complex& v = in[rowmajor(idx, hdims, r)];
            a[(size_t)li] = cld(v[0], v[1]);
        } else {
            // the redundant half: X[i] = conj(X[-i mod n])
            for (int d = 0; d < r; ++d) neg[d] = (p->n[d] - idx[d]) % p->n[d];
            const fftw_complex& v = in[rowmajor(neg, hdims, r)];
            a[(size_t)li] = cld(v[0], -(long double)v[1]);
        }
    }
    dft_block(a, p->n, r, FFTW_BACKWARD);
    for (long long li = 0; li < total; ++li) out[li] = (double)a[(size_t)li].real();
}

}  // namespace

extern "C" {

void* fftw_malloc(size_t n) {
    void* p = nullptr;
    if (posix_memalign(&p, 64, n ? n : 64) != 0) return nullptr;
    return p;
}
void fftw_free(void* p) { std::free(p); }
void fftw_destroy_plan(fftw_plan p) { delete p; }

void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out) {
    if (p && p->kind == C2C) exec_c2c(p, in, out);
}
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out) {
    if (p && p->kind == R2C) exec_r2c(p, in, out);
}
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out) {
    if (p && p->kind == C2R) exec_c2r(p, in, out);
}
void fftw_execute(const fftw_plan p) {
    if (!p) return;
    if (p->kind == C2C) exec_c2c(p, (fftw_complex*)p->in, (fftw_complex*)p->out);
    else if (p->kind == R2C) exec_r2c(p, (const double*)p->in, (fftw_complex*)p->out);
    else exec_c2r(p, (const fftw_complex*)p->in, (double*)p->out);
}

fftw_plan fftw_plan_dft(int rank, const int* n, fftw_complex* in, fftw_complex* out, int sign, unsigned) {
    return make_plan(C2C, rank, n, 1, in, nullptr, 1, 0, out, nullptr, 1, 0, sign);
}
fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags) {
    return fftw_plan_dft(1, &n, in, out, sign, flags);
}
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign, unsigned flags) {
    const int n[2] = {n0, n1};
    return fftw_plan_dft(2, n, in, out, sign, flags);
}
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign, unsigned flags) {
    const int n[3] = {n0, n1, n2};
    return fftw_plan_dft(3, n, in, out, sign, flags);
}
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out, unsigned) {
    const int n[3] = {n0, n1, n2};
    return make_plan(R2C, 3, n, 1, in, nullptr, 1, 0, out, nullptr, 1, 0, FFTW_FORWARD);
}
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out, unsigned) {
    const int n[3] = {n0, n1, n2};
    return make_plan(C2R, 3, n, 1, in, nullptr, 1, 0, out, nullptr, 1, 0, FFTW_BACKWARD);
}
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed, int istride,
                             int idist, fftw_complex* out, const int* onembed, int ostride, int odist, int sign,
                             unsigned) {
    return make_plan(C2C, rank, n, howmany, in, inembed, istride, idist, out, onembed, ostride, odist, sign);
}
void fftw_cleanup(void) {}
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int) {}
void fftw_cleanup_threads(void) {}

}  // extern "C"
