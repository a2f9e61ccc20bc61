// layout_io.cpp -- reference layout files, the benchmark layout generator and
// the reference bounds rule (host side of the drop-in boundary).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "frw_internal.h"
#include "layout_io.h"

namespace frw {

// Parser::parse + loadRectFromLine (CPU/Parser.cpp:15-50,89-125): lines are
// read with istream::getline into a 50-byte buffer, so a line of 50 or more
// characters ends the read (failbit) exactly as in the reference; every line
// containing "<<" closes a layer except the first; a line containing "rect"
// holds a header token and four numbers (other counts are undefined in the
// reference and rejected here); rects after the last delimiter are dropped.
frw_status parse_layout_file(const char *path, int layer, std::vector<double> *rects, int *nlayers) {
    rects->clear();
    if (nlayers) *nlayers = 0;
    std::ifstream file(path, std::ios::in);
    if (!file.is_open()) {
        set_error(std::string("cannot open layout file ") + path);
        return FRW_E_IO;
    }
    char line[50];
    bool first = true;
    int li = 0, lineno = 0;
    std::vector<double> cur;
    bool found = false;
    while (file.getline(line, sizeof(line))) {
        lineno++;
        if (strstr(line, "<<")) {
            if (first) {
                first = false;
                continue;
            }
            if (li == layer) {
                *rects = cur;
                found = true;
            }
            cur.clear();
            li++;
            continue;
        }
        if (strstr(line, "rect")) {
            std::istringstream ss{std::string(line)};
            std::string header;
            ss >> header;
            double v[5];
            int k = 0;
            while (k < 5 && ss >> v[k]) k++;
            if (k != 4) {
                set_error(std::string(path) + ":" + std::to_string(lineno) +
                          ": a rect line needs exactly 4 numbers");
                return FRW_E_IO;
            }
            cur.insert(cur.end(), v, v + 4);
        }
    }
    if (nlayers) *nlayers = li;
    if (!found) {
        set_error(std::string(path) + ": no layer " + std::to_string(layer) + " (" + std::to_string(li) +
                  " closed layers)");
        return FRW_E_ARG;
    }
    return FRW_OK;
}

// Parser::getLayerSize (CPU/Parser.cpp:51-87).
void reference_bounds(const double *r, int64_t n, double out[4]) {
    double lx = r[0], ty = r[1], rx = r[2], by = r[3];
    for (int64_t i = 1; i < n; i++) {
        const double *q = r + 4 * i;
        if (q[0] < lx) lx = q[0];
        if (q[1] < ty) ty = q[1];
        if (q[2] > rx) rx = q[2];
        if (q[3] > by) by = q[3];
    }
    bounds_from_extent(lx, ty, rx, by, out);
}

// The margin rule of Parser::getLayerSize (CPU/Parser.cpp:79-84): the
// bounding box grown on every side by int(0.01 * width) -- the width's
// margin on the y axis too, as the reference does.
void bounds_from_extent(double lx, double ty, double rx, double by, double out[4]) {
    const int add_w = (int)((rx - lx) * 0.01);
    out[0] = lx - add_w;
    out[1] = ty - add_w;
    out[2] = rx + add_w;
    out[3] = by + add_w;
}

namespace {
struct SplitMix {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    int64_t range(int64_t a, int64_t b) { return a + (int64_t)(next() % (uint64_t)(b - a + 1)); }
};
}  // namespace

frw_status generate_layout(uint64_t seed, int64_t n, double domain, int wmin, int wmax, double gap,
                           float *out) {
    if (n <= 0 || wmin < 1 || wmax < wmin || domain < wmax || gap < 0 || domain >= 16777216.0) {
        set_error("frw_generate_layout: bad arguments");
        return FRW_E_ARG;
    }
    const int64_t D = (int64_t)floor(domain);
    const double cs = wmax + ceil(gap) + 1.0;
    const int64_t nc = (int64_t)(D / cs) + 1;
    if (nc > 1 << 20) {
        set_error("frw_generate_layout: domain too large for the rejection grid");
        return FRW_E_ARG;
    }
    std::vector<int32_t> head((size_t)(nc * nc), -1), link((size_t)n, -1);  // per-cell lists
    SplitMix rng{seed};
    int64_t got = 0, tries = 0;
    while (got < n) {
        if (++tries > 64 * n + 1000) {
            set_error("frw_generate_layout: domain too crowded for the requested count");
            return FRW_E_ARG;
        }
        const int64_t w = rng.range(wmin, wmax), h = rng.range(wmin, wmax);
        const int64_t x0 = rng.range(0, D - w), y0 = rng.range(0, D - h);
        const int64_t x1 = x0 + w, y1 = y0 + h;
        const int64_t cx0 = std::max<int64_t>(0, (int64_t)((x0 - wmax - gap) / cs) - 1);
        const int64_t cx1 = std::min<int64_t>(nc - 1, (int64_t)((x1 + gap) / cs) + 1);
        const int64_t cy0 = std::max<int64_t>(0, (int64_t)((y0 - wmax - gap) / cs) - 1);
        const int64_t cy1 = std::min<int64_t>(nc - 1, (int64_t)((y1 + gap) / cs) + 1);
        bool ok = true;
        for (int64_t cy = cy0; cy <= cy1 && ok; cy++)
            for (int64_t cx = cx0; cx <= cx1 && ok; cx++)
                for (int32_t j = head[(size_t)(cy * nc + cx)]; j >= 0; j = link[(size_t)j]) {
                    const float *q = out + 4 * (int64_t)j;
                    const double g = std::max(std::max(q[0] - (double)x1, (double)x0 - q[2]),
                                              std::max(q[1] - (double)y1, (double)y0 - q[3]));
                    if (g < gap) {
                        ok = false;
                        break;
                    }
                }
        if (!ok) continue;
        float *o = out + 4 * got;
        o[0] = (float)x0;
        o[1] = (float)y0;
        o[2] = (float)x1;
        o[3] = (float)y1;
        const size_t c = (size_t)((int64_t)(y0 / cs) * nc + (int64_t)(x0 / cs));
        link[(size_t)got] = head[c];
        head[c] = (int32_t)got;
        got++;
    }
    return FRW_OK;
}

// The 3-D variant: integer corners uniform in [0, D)^2 x [0, Dz), edges
// uniform in [wmin, wmax] (z: [zmin, zmax]), accepted when the L-infinity gap
// to every accepted box is at least `gap` (a hash grid of cubes of side
// max edge + gap + 1 finds the neighbours).
frw_status generate_layout3(uint64_t seed, int64_t n, double domain, double zdomain, int wmin, int wmax, int zmin,
                            int zmax, double gap, float *out) {
    if (n <= 0 || n > INT32_MAX || wmin < 1 || wmax < wmin || zmin < 1 || zmax < zmin || domain < wmax ||
        zdomain < zmax || gap < 0 || domain >= 16777216.0 || zdomain >= 16777216.0) {
        set_error("frw3_generate_layout: bad arguments");
        return FRW_E_ARG;
    }
    const int64_t D = (int64_t)floor(domain), Dz = (int64_t)floor(zdomain);
    const int64_t emax = std::max(wmax, zmax);
    const double cs = emax + ceil(gap) + 1.0;
    const int64_t nc = (int64_t)(D / cs) + 1, ncz = (int64_t)(Dz / cs) + 1;
    if (nc * nc * ncz > (1ll << 26)) {
        set_error("frw3_generate_layout: domain too large for the rejection grid");
        return FRW_E_ARG;
    }
    std::vector<int32_t> head((size_t)(nc * nc * ncz), -1), link((size_t)n, -1);
    SplitMix rng{seed};
    int64_t got = 0, tries = 0;
    while (got < n) {
        if (++tries > 64 * n + 1000) {
            set_error("frw3_generate_layout: domain too crowded for the requested count");
            return FRW_E_ARG;
        }
        const int64_t w = rng.range(wmin, wmax), h = rng.range(wmin, wmax), d = rng.range(zmin, zmax);
        const int64_t x0 = rng.range(0, D - w), y0 = rng.range(0, D - h), z0 = rng.range(0, Dz - d);
        const int64_t lo[3] = {x0, y0, z0}, hi[3] = {x0 + w, y0 + h, z0 + d}, ncs[3] = {nc, nc, ncz};
        int64_t c0[3], c1[3];
        for (int c = 0; c < 3; c++) {
            c0[c] = std::max<int64_t>(0, (int64_t)((lo[c] - emax - gap) / cs) - 1);
            c1[c] = std::min<int64_t>(ncs[c] - 1, (int64_t)((hi[c] + gap) / cs) + 1);
        }
        bool ok = true;
        for (int64_t cz = c0[2]; cz <= c1[2] && ok; cz++)
            for (int64_t cy = c0[1]; cy <= c1[1] && ok; cy++)
                for (int64_t cx = c0[0]; cx <= c1[0] && ok; cx++)
                    for (int32_t j = head[(size_t)((cz * nc + cy) * nc + cx)]; j >= 0; j = link[(size_t)j]) {
                        const float *q = out + 6 * (int64_t)j;
                        double g = -INFINITY;
                        for (int c = 0; c < 3; c++)
                            g = std::max(g, std::max(q[c] - (double)hi[c], (double)lo[c] - q[3 + c]));
                        if (g < gap) {
                            ok = false;
                            break;
                        }
                    }
        if (!ok) continue;
        float *o = out + 6 * got;
        for (int c = 0; c < 3; c++) {
            o[c] = (float)lo[c];
            o[3 + c] = (float)hi[c];
        }
        const size_t cell = (size_t)(((int64_t)(z0 / cs) * nc + (int64_t)(y0 / cs)) * nc + (int64_t)(x0 / cs));
        link[(size_t)got] = head[cell];
        head[cell] = (int32_t)got;
        got++;
    }
    return FRW_OK;
}

frw_status write_layout(const char *path, const float *r, int64_t n, const char *name) {
    FILE *f = fopen(path, "w");
    if (!f) {
        set_error(std::string("cannot write ") + path);
        return FRW_E_IO;
    }
    const char *nm = name ? name : "layer";
    fprintf(f, "<< %s >>\n", nm);
    for (int64_t i = 0; i < n; i++)
        fprintf(f, "rect %.9g %.9g %.9g %.9g\n", r[4 * i], r[4 * i + 1], r[4 * i + 2], r[4 * i + 3]);
    fprintf(f, "<< end >>\n");
    if (fclose(f) != 0) {
        set_error(std::string("write failed: ") + path);
        return FRW_E_IO;
    }
    return FRW_OK;
}

}  // namespace frw
