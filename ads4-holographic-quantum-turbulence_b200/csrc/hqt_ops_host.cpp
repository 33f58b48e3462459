// hqt_ops_host.cpp -- host-side operator construction (FP64).
#include "hqt_ops_host.h"

#include <cmath>


namespace hqt {

void chebdif_row(int N, int i, double *row) {
    const double pi = 3.14159265358979323846;
    auto th = [&](int k) { return k * pi / (N - 1); };
    // DX(i,j) = 2 sin((th_j+th_i)/2) sin((th_j-th_i)/2); rows i >= N/2 use
    // the flipped form -DX(N-1-i, N-1-j)
    auto dx_raw = [&](int r, int c) {
        return 2.0 * std::sin(th(c) / 2 + th(r) / 2) * std::sin(th(c) / 2 - th(r) / 2);
    };
    const int n1 = N / 2;
    double rowsum = 0.0;
    for (int j = 0; j < N; ++j) {
        if (j == i) continue;
        const double dx = (i < n1) ? dx_raw(i, j) : -dx_raw(N - 1 - i, N - 1 - j);
        double c = ((i + j) % 2 == 0) ? 1.0 : -1.0;
        if (i == 0 || i == N - 1) c *= 2.0;
        if (j == 0 || j == N - 1) c /= 2.0;
        const double v = (1.0 / dx) * c;
        row[j] = v;
        rowsum += v;
    }
    row[i] = -rowsum;
}

void chebdif_host(int N, std::vector<double> &x, std::vector<double> &D) {
    x.assign(N, 0.0);
    D.assign((size_t)N * N, 0.0);
    const double pi = 3.14159265358979323846;
    std::vector<double> th(N);
    for (int k = 0; k < N; ++k) {
        th[k] = k * pi / (N - 1);
        x[k] = std::sin(pi * (N - 1 - 2 * k) / (2.0 * (N - 1)));
    }
    // DX(i,j) = 2 sin((th_j+th_i)/2) sin((th_j-th_i)/2), flipped lower half
    std::vector<double> DX((size_t)N * N);
    auto dx_raw = [&](int i, int j) {
        return 2.0 * std::sin(th[j] / 2 + th[i] / 2) * std::sin(th[j] / 2 - th[i] / 2);
    };
    const int n1 = N / 2, n2 = (N + 1) / 2;
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            double v;
            if (i < n1)
                v = dx_raw(i, j);
            else  // -flipud(fliplr(DX(1:n2,:))) row i -> source row N-1-i, col N-1-j
                v = -dx_raw(N - 1 - i, N - 1 - j);
            (void)n2;
            DX[(size_t)i * N + j] = (i == j) ? 1.0 : v;
        }
    for (int i = 0; i < N; ++i) {
        double rowsum = 0.0;
        for (int j = 0; j < N; ++j) {
            if (i == j) continue;
            double c = ((i + j) % 2 == 0) ? 1.0 : -1.0;
            if (i == 0 || i == N - 1) c *= 2.0;
            if (j == 0 || j == N - 1) c /= 2.0;
            const double v = (1.0 / DX[(size_t)i * N + j]) * c;
            D[(size_t)i * N + j] = v;
            rowsum += v;
        }
        D[(size_t)i * N + i] = -rowsum;
    }
}

bool invert_host(int n, const std::vector<double> &A, std::vector<double> &inv) {
    std::vector<long double> M((size_t)n * 2 * n, 0.0L);
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) M[(size_t)i * 2 * n + j] = A[(size_t)i * n + j];
        M[(size_t)i * 2 * n + n + i] = 1.0L;
    }
    for (int c = 0; c < n; ++c) {
        int piv = c;
        long double best = std::fabs(M[(size_t)c * 2 * n + c]);
        for (int r = c + 1; r < n; ++r) {
            const long double v = std::fabs(M[(size_t)r * 2 * n + c]);
            if (v > best) {
                best = v;
                piv = r;
            }
        }
        if (best == 0.0L) return false;
        if (piv != c)
            for (int j = 0; j < 2 * n; ++j)
                std::swap(M[(size_t)c * 2 * n + j], M[(size_t)piv * 2 * n + j]);
        const long double d = M[(size_t)c * 2 * n + c];
        for (int j = 0; j < 2 * n; ++j) M[(size_t)c * 2 * n + j] /= d;
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const long double f = M[(size_t)r * 2 * n + c];
            if (f == 0.0L) continue;
            for (int j = 0; j < 2 * n; ++j)
                M[(size_t)r * 2 * n + j] -= f * M[(size_t)c * 2 * n + j];
        }
    }
    inv.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) inv[(size_t)i * n + j] = (double)M[(size_t)i * 2 * n + n + j];
    return true;
}

FFTPlan make_plan(int n) {
    FFTPlan p{};
    p.n = n;
    int m = n;
    int p2 = 0;
    while (m % 2 == 0) {
        m /= 2;
        ++p2;
    }
    std::vector<int> rad;
    // power-of-two part: ceil(p2/3) passes, bits spread evenly (8, 4, 2); a
    // radix-16 pass held 16 complex values in registers and spilled in FP64
    if (p2 > 0) {
        const int npass = (p2 + 2) / 3;
        int left = p2;
        for (int i = 0; i < npass; ++i) {
            const int bits = (left + (npass - i) - 1) / (npass - i);
            rad.push_back(1 << bits);
            left -= bits;
        }
    }
    // odd part: prime factors, ascending
    for (int f = 3; (long long)f * f <= m; f += 2)
        while (m % f == 0) {
            rad.push_back(f);
            m /= f;
        }
    if (m > 1) rad.push_back(m);
    p.npass = (int)rad.size();
    int ns = 1;
    for (int i = 0; i < p.npass && i < kMaxPass; ++i) {
        p.radix[i] = rad[i];
        p.ns[i] = ns;
        ns *= rad[i];
    }
    return p;
}

std::vector<double2> make_roots(int n) {
    std::vector<double2> r(n);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int q = 0; q < n; ++q) {
        const long double a = 2.0L * pi * (long double)q / (long double)n;
        r[q].x = (double)std::cos(a);
        r[q].y = (double)(-std::sin(a));
    }
    return r;
}

void make_radix_tables(std::vector<double> &c, std::vector<double> &s) {
    c.clear();
    s.clear();
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < kNumTabRadices; ++i) {
        const int R = kTabRadices[i];
        for (int t = 0; t < R; ++t) {
            const long double a = 2.0L * pi * (long double)t / (long double)R;
            c.push_back((double)std::cos(a));
            s.push_back((double)std::sin(a));
        }
    }
}

void make_big_tables(std::vector<double> &c, std::vector<double> &s) {
    static const int primes[] = {17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61};
    c.clear();
    s.clear();
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int R : primes)
        for (int t = 0; t < R; ++t) {
            const long double a = 2.0L * pi * (long double)t / (long double)R;
            c.push_back((double)std::cos(a));
            s.push_back((double)std::sin(a));
        }
}

static int matlab_round_pos(double v) { return (int)std::floor(v + 0.5); }

void filter_band(int n, int &lo, int &hi) {
    lo = matlab_round_pos((double)matlab_round_pos((double)n / 3.0));
    hi = matlab_round_pos((double)n / 3.0 * 2.0);
}

}  // namespace hqt
