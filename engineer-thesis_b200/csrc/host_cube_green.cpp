// host_cube_green.cpp -- unit-cube Green's function tables (host, FP64).
//
// The landing density on the surface of the cube [0,1]^3 seen from its
// centre, per face (the face z = 0 shown; the six faces are parametrised by
// (eta, dzeta) in [k, k+1)^2, green/green.h:66-70):
//   K(x, y) = 4 sum_{m,n odd} s_m s_n sin(m pi x) sin(n pi y) / (2 cosh(g_mn / 2)),
//   g_mn = pi sqrt(m^2 + n^2),  s_k = sin(k pi / 2),
// and its gradient with respect to the centre (normal part with
// 1/(2 sinh(g/2)) and a factor g_mn, tangential parts with cos(k pi / 2) and
// a factor k pi), both truncated at m, n <= 20 (NTERMS, green/green.cpp:21).
// The table is the reference's precompute_unit_cube_green
// (green/green.cpp:392-431): samples at the centres of an n x n grid on each
// face, the running sum of g times the cell area normalised to 1.
//
// It has to be bit-identical to the reference's table, so every sample is
// the same sequence of correctly rounded operations on the same libm
// results; only the work is shared: each sine and exponential the series
// needs is evaluated once per distinct argument (the 6 n sample abscissae
// and the 20 x 20 (m, n) pairs) instead of once per sample, which makes a
// 50 x 50 table about 30x cheaper.  Multiplying by +-1 is exact, so the sign
// factors are applied where convenient.  The host compiler runs with
// -ffp-contract=off.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "frw3d_internal.h"

namespace frw {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kTerms = 20;

inline double sgn_of(unsigned k) { return ((k >> 1) & 1u) ? -1.0 : 1.0; }

struct Series {
    double c[kTerms + 1][kTerms + 1];   // 1/(2 cosh(g/2)) as q (1 - q^2) / (1 - q^4)
    double c1[kTerms + 1][kTerms + 1];  // 1/(2 sinh(g/2)) as q (1 + q^2) / (1 - q^4)
    double r[kTerms + 1][kTerms + 1];   // sqrt(m^2 + n^2)
    Series() {
        for (unsigned m = 1; m <= kTerms; m++)
            for (unsigned n = 1; n <= kTerms; n++) {
                const double rt = sqrt((double)(m * m + n * n));
                const double e = -0.5 * rt * kPi;
                const double q = exp(e);
                const double den = 1.0 - exp(4.0 * e);
                c[m][n] = q * (1.0 - q * q) / den;
                c1[m][n] = q * (1.0 + q * q) / den;
                r[m][n] = rt;
            }
    }
};

const Series &series() {
    static const Series s;
    return s;
}

int face_of(double eta, double a) {
    return eta < a ? 0 : eta < 2 * a ? 1 : eta < 3 * a ? 2 : eta < 4 * a ? 3 : eta < 5 * a ? 4 : 5;
}

// The series of K at (eta, dzeta) without its factor 4/a^2, from sines of
// the scaled abscissae: sm[m] = sin(m es), sn[n] = sin(n zs) for odd m, n.
double green_sum(const double *sm, const double *sn) {
    const Series &S = series();
    double acc = 0.0;
    for (unsigned m = 1; m <= kTerms; m += 2) {
        const double sin_m = sgn_of(m) * sm[m];
        for (unsigned n = 1; n <= kTerms; n += 2) acc += sgn_of(n) * S.c[m][n] * sn[n] * sin_m;
    }
    return acc;
}

// Normal (A) and tangential (B along the first axis, C along the second)
// sums from sines of the face-local scaled abscissae, m, n = 1..20.
void grad_from(const double *sm, const double *sn, double *A, double *B, double *C) {
    const Series &S = series();
    double a = 0.0, b = 0.0, c = 0.0;
    for (unsigned m = 1; m <= kTerms; m++) {
        const double sin_m = sm[m];
        for (unsigned n = 1; n <= kTerms; n++) {
            const double s = sgn_of(m) * sgn_of(n);
            if (n & 1) {
                if (m & 1) a += s * (S.r[m][n] * S.c1[m][n] * sn[n] * sin_m);
                else b += s * (m * S.c[m][n] * sn[n] * sin_m);
            } else if (m & 1) {
                c += s * (n * S.c[m][n] * sn[n] * sin_m);
            }
        }
    }
    *A = a;
    *B = b;
    *C = c;
}

// -grad K on face k from the sums, axis signs of the face parametrisation:
// faces 0 (u,v,0) 1 (1,u,v) 2 (1-v,1,u) 3 (1-u,1-v,1) 4 (0,1-u,1-v) 5 (v,0,1-u).
void place_grad(int k, double A, double B, double C, double scale, double *dg) {
    double x, y, z;
    switch (k) {
    case 0: x = B; y = C; z = -A; break;
    case 1: x = A; y = B; z = C; break;
    case 2: x = -B; y = A; z = C; break;
    case 3: x = -B; y = -C; z = A; break;
    case 4: x = -A; y = -B; z = -C; break;
    default: x = B; y = -A; z = -C; break;
    }
    dg[0] = x * scale;
    dg[1] = y * scale;
    dg[2] = z * scale;
}

struct CubeTable {
    int n = 0;
    std::vector<double> g, dx, dy, dz, intg;
};

std::shared_ptr<const CubeTable> make_table(int n) {
    auto T = std::make_shared<CubeTable>();
    const size_t N = (size_t)n, nb = 6 * N * N, na = 6 * N;
    T->n = n;
    T->g.resize(nb);
    T->dx.resize(nb);
    T->dy.resize(nb);
    T->dz.resize(nb);
    T->intg.resize(nb + 1);
    const double delta = 1.0 / n;
    // Abscissa t (t = 0 .. 6n-1) is (t + 1/2) delta for eta and dzeta alike;
    // sg[t][m] = sin(m pi val / 1), sl[t][m] = sin(m pi (val - k) / 1) with k
    // the face of val.
    std::vector<double> sg((kTerms + 1) * na), sl((kTerms + 1) * na);
    std::vector<int> face(na);
    for (size_t t = 0; t < na; t++) {
        const double val = (t + 0.5) * delta;
        const int k = face_of(val, 1.0);
        face[t] = k;
        const double es = kPi * val / 1.0;
        const double el = kPi * (val - k * 1.0) / 1.0;
        for (unsigned m = 1; m <= kTerms; m++) {
            sg[t * (kTerms + 1) + m] = sin((double)m * es);
            sl[t * (kTerms + 1) + m] = sin(m * el);
        }
    }
    const double scale = -4.0 * kPi / (1.0 * 1.0 * 1.0);
    double prev_int = 0.0, prev_g = 0.0;
    for (size_t k = 0; k < 6; k++)
        for (size_t i = k * N; i < (k + 1) * N; i++)
            for (size_t j = 0; j < N; j++) {
                const size_t tz = k * N + j, idx = i * N + j;
                const double *ge = &sg[i * (kTerms + 1)], *gz = &sg[tz * (kTerms + 1)];
                const double *le = &sl[i * (kTerms + 1)], *lz = &sl[tz * (kTerms + 1)];
                const double gv = green_sum(ge, gz) * (4 / (1.0 * 1.0));
                const int f = face[i];
                double A, B, C, d[3];
                if (f == 2 || f == 5) grad_from(lz, le, &A, &B, &C);
                else grad_from(le, lz, &A, &B, &C);
                place_grad(f, A, B, C, scale, d);
                T->g[idx] = gv;
                T->dx[idx] = d[0];
                T->dy[idx] = d[1];
                T->dz[idx] = d[2];
                const double cum = prev_int + prev_g * delta * delta;
                T->intg[idx] = cum;
                prev_int = cum;
                prev_g = gv;
            }
    T->intg[nb] = prev_int + prev_g * delta * delta;
    const double alpha = 1.0 / T->intg[nb];
    for (size_t i = 0; i <= nb; i++) T->intg[i] *= alpha;
    return T;
}

std::shared_ptr<const CubeTable> table_for(int n) {
    static std::mutex mu;
    static std::map<int, std::shared_ptr<const CubeTable>> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(n);
    if (it != cache.end()) return it->second;
    auto T = make_table(n);
    cache[n] = T;
    return T;
}

}  // namespace

bool cube_green_table(int n, double *g, double *dgdx, double *dgdy, double *dgdz, double *intg) {
    if (n < 1 || n > FRW3_NSAMPLE_MAX) return false;
    auto T = table_for(n);
    const size_t nb = T->g.size();
    if (g) memcpy(g, T->g.data(), nb * sizeof(double));
    if (dgdx) memcpy(dgdx, T->dx.data(), nb * sizeof(double));
    if (dgdy) memcpy(dgdy, T->dy.data(), nb * sizeof(double));
    if (dgdz) memcpy(dgdz, T->dz.data(), nb * sizeof(double));
    if (intg) memcpy(intg, T->intg.data(), (nb + 1) * sizeof(double));
    return true;
}

// green_cube(a, eta, dzeta) at one point (green/green.cpp:232-267).
double cube_green_point(double a, double eta, double dzeta) {
    const double es = kPi * eta / a, zs = kPi * dzeta / a;
    double sm[kTerms + 1], sn[kTerms + 1];
    for (unsigned m = 1; m <= kTerms; m += 2) {
        sm[m] = sin((double)m * es);
        sn[m] = sin((double)m * zs);
    }
    return green_sum(sm, sn) * (4 / (a * a));
}

// deriv_green_cube(dg, a, eta, dzeta) at one point (green/green.cpp:311-388).
void cube_deriv_point(double *dg, double a, double eta, double dzeta) {
    const int k = face_of(eta, a);
    const double es = kPi * (eta - k * a) / a, zs = kPi * (dzeta - k * a) / a;
    double se[kTerms + 1], sz[kTerms + 1], A, B, C;
    for (unsigned m = 1; m <= kTerms; m++) {
        se[m] = sin(m * es);
        sz[m] = sin(m * zs);
    }
    if (k == 2 || k == 5) grad_from(sz, se, &A, &B, &C);
    else grad_from(se, sz, &A, &B, &C);
    place_grad(k, A, B, C, -4.0 * kPi / (a * a * a), dg);
}

bool cube_walk_tables(int n, uint32_t *thr, uint16_t *guide, double *w, double *offs) {
    if (n < 1 || n > FRW3_NSAMPLE_MAX) return false;
    auto T = table_for(n);
    const int nb = 6 * n * n;
    std::vector<uint64_t> t64(nb);
    for (int b = 0; b < nb; b++) {
        t64[b] = (uint64_t)ceil(ldexp(T->intg[b], 32));
        if (t64[b] > 0xFFFFFFFFull) return false;  // a bin of zero mass before the end
    }
    if (thr)
        for (int b = 0; b < nb; b++) thr[b] = (uint32_t)t64[b];
    if (guide)
        for (int k = 0; k < (1 << kGuide3Bits); k++) {
            const uint64_t x = (uint64_t)k << (32 - kGuide3Bits);
            // last bin with threshold <= x (thresholds nondecreasing, thr[0] = 0)
            const int b = (int)(std::upper_bound(t64.begin(), t64.end(), x) - t64.begin()) - 1;
            guide[k] = (uint16_t)std::max(b, 0);
        }
    if (w) {
        const double area = 1.0 / ((double)n * (double)n);
        for (int b = 0; b < nb; b++) {
            const double pi_b = T->intg[b + 1] - T->intg[b];
            const double f = pi_b > 0 ? area / pi_b : 0.0;
            w[3 * b] = T->dx[b] * f;
            w[3 * b + 1] = T->dy[b] * f;
            w[3 * b + 2] = T->dz[b] * f;
        }
    }
    if (offs)
        for (int i = 0; i < n; i++) offs[i] = (double)(2 * i + 1 - n) / (double)n;
    return true;
}

}  // namespace frw
