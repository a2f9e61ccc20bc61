// host_green.cpp -- unit-square Green's function tables (host, FP64).
//
// The walk samples the boundary of each transition square from the surface
// Green's function of a square seen from its centre.  For [0,1]^2 with data
// on one side and zero on the others, separation of variables gives the
// Poisson kernel at the centre
//     K(t) = 2 sum_{n odd} (-1)^((n-1)/2) c_n sin(n pi t),
//     c_n  = sinh(n pi/2) / sinh(n pi) = q (1 - q^2) / (1 - e^{-2 pi n}),  q = e^{-n pi/2},
// t in [0,1] along the side.  Over the perimeter parameter eta in [0,4) the
// side index k flips the sign of sin(n pi eta) for odd n, which the side sign
// (-1)^k undoes.  The table samples eta_i = (i + 1/2) * 4/N with the series
// truncated at n <= 19, the sampling and truncation of the reference's
// precompute_unit_square_green (green/green.cpp:27-54,125-152); the
// cumulative sum is accumulated in the same order so the CDF the walks
// compare uniforms against is bit-identical to the reference's.
//
// The first-hop capacitance weight needs the gradient of K with respect to
// the source point (at the centre): normal part (towards the side)
//     N(t) = 2 pi sum_{n odd}  (-1)^((n-1)/2) n ch_n sin(n pi t),  ch_n = cosh(n pi/2)/sinh(n pi),
// tangential part (along the side)
//     T(t) = 2 pi sum_{n even} (-1)^(n/2) n c_n sin(n pi t),
// summed to n = 80 (terms decay like n e^{-n pi/2}).  Bin i of the reference's
// perimeter mapping lands on segment i-1 of its side (corners for i = 0 mod
// N/4), so the weight of bin i is evaluated there:
//     W_i = grad K(landing point) * (1/(N/4)) / pi_i,   pi_i = intg[i+1] - intg[i],
// which makes  (1/a) E[W_i . n phi(x_i)]  the quadrature of dphi/dn at the
// centre of a square of side a.
#include <math.h>
#include <stdint.h>

#include "frw_internal.h"

namespace frw {
namespace {

double kernel_at(double eta) {
    const double pi = 3.14159265358979323846;
    const double ph = pi * eta / 1.0;
    double acc = 0.0, sgn = 1.0;
    for (uint64_t n = 1; n <= 20; n += 2) {
        const double q = exp(-0.5 * n * pi);
        const double den = 1.0 - exp(-2.0 * pi * n);
        acc += sgn * (q * (1.0 - q * q) / den) * sin(n * ph);
        sgn *= -1;
    }
    const int side = eta <= 1.0 ? 0 : eta <= 2.0 ? 1 : eta <= 3.0 ? 2 : 3;
    return acc * ((side & 1) ? -2.0 / 1.0 : 2.0 / 1.0);
}

void kernel_grad(double t, double *nrm, double *tan) {
    const double pi = 3.14159265358979323846;
    double sn = 0.0, st = 0.0;
    for (int n = 1; n <= 80; n++) {
        const double q = exp(-0.5 * n * pi);
        const double den = 1.0 - exp(-2.0 * pi * n);
        const double s = sin(n * pi * t);
        const double sg = ((n >> 1) & 1) ? -1.0 : 1.0;
        if (n & 1) sn += sg * n * (q * (1.0 + q * q) / den) * s;
        else st += sg * n * (q * (1.0 - q * q) / den) * s;
    }
    *nrm = 2.0 * pi * sn;
    *tan = 2.0 * pi * st;
}

}  // namespace

void green_tables(double *g, double *intg, double *wx, double *wy) {
    const int N = FRW_NSAMPLE;
    const double d_eta = 4.0 / N;
    double gl[FRW_NSAMPLE], cl[FRW_NSAMPLE + 1];
    for (uint64_t i = 0; i < (uint64_t)N; i++) gl[i] = kernel_at((i + 0.5) * d_eta);
    cl[0] = 0.0;
    for (uint64_t i = 1; i <= (uint64_t)N; i++) cl[i] = cl[i - 1] + gl[i - 1] * d_eta;
    const double alpha = 1.0 / cl[N];
    for (int i = 0; i <= N; i++) cl[i] *= alpha;
    if (g)
        for (int i = 0; i < N; i++) g[i] = gl[i];
    if (intg)
        for (int i = 0; i <= N; i++) intg[i] = cl[i];
    if (wx && wy) {
        // screen axes (y down), clockwise from the top-left corner
        static const double along[4][2] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
        static const double outw[4][2] = {{0, -1}, {1, 0}, {0, 1}, {-1, 0}};
        const int nside = N / 4;
        for (int i = 0; i < N; i++) {
            const int s = i / nside, j = i % nside;
            if (j == 0) {
                wx[i] = wy[i] = 0.0;
                continue;
            }
            double nr, tg;
            kernel_grad(((j - 1) + 0.5) / nside, &nr, &tg);
            const double f = (1.0 / nside) / (cl[i + 1] - cl[i]);
            wx[i] = (tg * along[s][0] + nr * outw[s][0]) * f;
            wy[i] = (tg * along[s][1] + nr * outw[s][1]) * f;
        }
    }
}

}  // namespace frw
