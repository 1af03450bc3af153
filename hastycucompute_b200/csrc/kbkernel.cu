// Host side of the Kaiser-Bessel kernel: beta, I0, phi, its Fourier transform, and the
// Chebyshev fit of the per-tap polynomials the device evaluates.
#include <cmath>
#include <cstring>

#include "kbkernel.cuh"

namespace hb {

double kb_beta(int w, double sigma) {
    // beta = pi * sqrt((w/sigma)^2 (sigma - 1/2)^2 - 0.8)
    double a = (double)w / sigma * (sigma - 0.5);
    double v = a * a - 0.8;
    return v > 0 ? M_PI * std::sqrt(v) : 0.0;
}

double bessel_i0(double x) {
    // I0(x) = sum_k ((x/2)^k / k!)^2
    double q = 0.25 * x * x, term = 1.0, sum = 1.0;
    for (int k = 1; k < 500; ++k) {
        term *= q / ((double)k * (double)k);
        sum += term;
        if (term < 1e-18 * sum) break;
    }
    return sum;
}

double kb_phi(double z, int w, double beta) {
    double r = 2.0 * z / (double)w;
    double a = 1.0 - r * r;
    if (a < 0) return 0.0;
    return bessel_i0(beta * std::sqrt(a)) / bessel_i0(beta);
}

double kb_phihat(double xi, int w, double beta) {
    // int_{-w/2}^{w/2} I0(beta sqrt(1-(2z/w)^2)) e^{-2 pi i xi z} dz
    //   = w sinh(sqrt(beta^2 - a^2)) / sqrt(beta^2 - a^2),  a = pi w xi
    // (sin form when a > beta), divided by I0(beta) like phi.
    double a = M_PI * (double)w * xi;
    double d = beta * beta - a * a;
    double v;
    if (d > 1e-12) {
        double s = std::sqrt(d);
        v = std::sinh(s) / s;
    } else if (d < -1e-12) {
        double s = std::sqrt(-d);
        v = std::sin(s) / s;
    } else {
        v = 1.0;
    }
    return (double)w * v / bessel_i0(beta);
}

double kb_fit(KbPoly* p, int w, double beta) {
    std::memset(p, 0, sizeof(KbPoly));
    p->w = w;
    p->hw = 0.5f * (float)w;
    double worst = 0.0;
    for (int deg = (w + 2 < kMaxDeg ? w + 2 : kMaxDeg); deg <= kMaxDeg; ++deg) {
        const int n = deg + 1;
        worst = 0.0;
        for (int d = 0; d < w; ++d) {
            // Chebyshev coefficients of f(s) = phi(d - w/2 + (s+1)/2) on s in [-1,1].
            double fk[kMaxDeg + 1], a[kMaxDeg + 1] = {0};
            for (int k = 0; k < n; ++k) {
                double s = std::cos(M_PI * (k + 0.5) / n);
                fk[k] = kb_phi((double)d - 0.5 * w + 0.5 * (s + 1.0), w, beta);
            }
            for (int j = 0; j < n; ++j) {
                double acc = 0;
                for (int k = 0; k < n; ++k) acc += fk[k] * std::cos(M_PI * j * (k + 0.5) / n);
                a[j] = acc * 2.0 / n;
            }
            a[0] *= 0.5;
            // Chebyshev -> monomial: T_0 = 1, T_1 = s, T_{j+1} = 2 s T_j - T_{j-1}.
            double tprev[kMaxDeg + 2] = {0}, tcur[kMaxDeg + 2] = {0}, tnext[kMaxDeg + 2];
            double mono[kMaxDeg + 1] = {0};
            tprev[0] = 1.0;
            mono[0] += a[0];
            if (n > 1) {
                tcur[1] = 1.0;
                mono[1] += a[1];
            }
            for (int j = 2; j < n; ++j) {
                for (int m = 0; m <= kMaxDeg + 1; ++m) {
                    double v = -tprev[m];
                    if (m > 0) v += 2.0 * tcur[m - 1];
                    tnext[m] = v;
                }
                for (int m = 0; m <= deg; ++m) mono[m] += a[j] * tnext[m];
                std::memcpy(tprev, tcur, sizeof(tcur));
                std::memcpy(tcur, tnext, sizeof(tnext));
            }
            for (int m = 0; m <= deg; ++m) p->coef[d][m] = (float)mono[m];
            // Check in double on a dense grid.
            for (int q = 0; q <= 64; ++q) {
                double s = -1.0 + 2.0 * q / 64.0;
                double acc = mono[deg];
                for (int m = deg - 1; m >= 0; --m) acc = acc * s + mono[m];
                double ex = kb_phi((double)d - 0.5 * w + 0.5 * (s + 1.0), w, beta);
                if (q == 0 && d == 0) continue;  // s=-1 of tap 0 is the support edge
                worst = std::fmax(worst, std::fabs(acc - ex));
            }
        }
        p->deg = deg;
        if (worst < 1e-9) break;
    }
    return worst;
}

}  // namespace hb
