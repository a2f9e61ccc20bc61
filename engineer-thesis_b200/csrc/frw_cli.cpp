// frw_cli.cpp -- command-line front end with the reference's flags
// (randomWalk/main.cpp:25-126, defines.h:30-40):
//   -S/--source <file>  -I/--iterations <n>  -O/--object <id>  -L/--layer <k>
//   -G/--GPU (accepted; the device path is the only path)  -M/--measure  --help
// Extra flags: --seed <u64>, --device <k>, --uniform (uniform start and
// capacitance weights), --offset <d> (Gaussian surface = target grown by d),
// --scale <f> (reference scaled surface, default 1.5), --exact-perimeter,
// --cap (print the capacitance row), --hist <file> (histogram file name;
// default "<unixtime>wyniki.txt" as the reference writes), --json (one JSON
// result record on stdout after the reference's two lines), --3d
// <z0:z1,...> (3-D walk, include/frw3d.h: every layer of the file extruded to
// its z range, -O a box index in layer order, --offset the Gaussian offset,
// default 1; the capacitance row is that of the 3-D layout).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <chrono>
#include <string>
#include <vector>

#include "../../include/frw.h"
#include "../../include/frw3d.h"

static const char *kHelp =
    "\t-S\t--source\t\tlayout file\n"
    "\t-M\t--measure\t\tprint timings\n"
    "\t-O\t--object\t\ttarget rect id\n"
    "\t-I\t--iterations\t\tnumber of walks\n"
    "\t-G\t--GPU\t\t\t(accepted; walks always run on the GPU)\n"
    "\t-L\t--layer\t\t\tlayer number\n"
    "\t\t--seed <u64> --device <k> --uniform --offset <d> --scale <f>\n"
    "\t\t--exact-perimeter --cap --hist <file> --json\n"
    "\t\t--3d <z0:z1,...>\t3-D walk, layer k extruded to the k-th z range\n"
    "\t\t--help\t\t\tthis text\n"
    "\tDefaults: -I 1000 -O 10 -S ../tests/test -L 0\n";

// "z0:z1,z0:z1,..." -> ranges; false on a malformed list.
static bool parse_ranges(const std::string &s, std::vector<double> *z0, std::vector<double> *z1) {
    size_t i = 0;
    while (i < s.size()) {
        size_t j = s.find(',', i);
        if (j == std::string::npos) j = s.size();
        const std::string part = s.substr(i, j - i);
        const size_t c = part.find(':');
        if (c == std::string::npos) return false;
        char *e1 = nullptr, *e2 = nullptr;
        const std::string a = part.substr(0, c), b = part.substr(c + 1);
        const double lo = strtod(a.c_str(), &e1), hi = strtod(b.c_str(), &e2);
        if (a.empty() || b.empty() || *e1 || *e2) return false;
        z0->push_back(lo);
        z1->push_back(hi);
        i = j + 1;
    }
    return !z0->empty();
}

// The 3-D run: the same two lines, histogram, capacitance row and JSON
// record as the 2-D run, over the extruded layout.
static int run3d(const std::string &path, const std::string &zspec, long long iters, long long object, int device,
                 unsigned long long seed, double offset, bool measure, bool cap, bool json, std::string hist) {
    std::vector<double> z0, z1;
    if (!parse_ranges(zspec, &z0, &z1)) {
        fprintf(stderr, "--3d needs z0:z1[,z0:z1...]\n");
        return 2;
    }
    auto t0 = std::chrono::steady_clock::now();
    frw3_layout *L = nullptr;
    if (frw3_layout_from_file(path.c_str(), z0.data(), z1.data(), (int)z0.size(), nullptr, 0.0, device, &L) !=
        FRW_OK) {
        fprintf(stderr, "error: %s\n", frw_last_error());
        return 1;
    }
    frw3_layout_info info;
    frw3_layout_info_get(L, &info);
    if (object < 0 || object >= info.n) {
        fprintf(stderr, "Incorrect args! (object %lld of %lld boxes)\n", object, (long long)info.n);
        frw3_layout_destroy(L);
        return 2;
    }
    frw3_opts o;
    frw3_opts_default(&o);
    if (offset > 0) o.gauss_offset = offset;
    std::vector<int64_t> cond(info.n);
    std::vector<uint64_t> hits(info.n);
    std::vector<double> c(info.n), se(info.n);
    frw3_result r{};
    r.capacity = info.n;
    r.conductor = cond.data();
    r.hits = hits.data();
    r.cap = c.data();
    r.cap_se = se.data();
    if (frw3_walk(L, object, (uint64_t)iters, seed, &o, &r, nullptr) != FRW_OK) {
        fprintf(stderr, "error: %s\n", frw_last_error());
        frw3_layout_destroy(L);
        return 1;
    }
    auto t1 = std::chrono::steady_clock::now();
    std::vector<float> q(6 * info.n);
    frw3_layout_boxes(L, q.data());
    if (hist.empty()) hist = std::to_string((unsigned long)time(nullptr)) + "wyniki.txt";
    FILE *f = fopen(hist.c_str(), "w");
    if (f) {
        fprintf(f, "[GPU 3D]\n");
        if (r.escaped)
            fprintf(f, "Ile scie\xc5\xbc" "ek wysz\xc5\x82o poza granice: %g%%\n", (float)r.escaped / (float)iters * 100);
        for (int64_t k = 0; k < r.n_entries && k < r.capacity; k++) {
            const float *b = &q[6 * cond[k]];
            fprintf(f, "%g %g %g %g %g %g: %g%%\n", b[0], b[1], b[2], b[3], b[4], b[5],
                    ((float)hits[k] / (float)iters) * 100);
        }
        fclose(f);
        printf("Wynik zapisany do %s\n", hist.c_str());
    }
    printf("[GPU] Ile sciezek trafi\xc5\x82o do innego elementu: %f%%\n", r.fraction_other * 100.);
    printf("Czas wykonania: %lld ms\n",
           (long long)std::chrono::duration_cast<std::chrono::milliseconds>(t1 - t0).count());
    if (measure)
        printf("grid build %.3f ms (%d x %d x %d cells, %.1f per list); walk kernel %.3f ms; %.1f hops/walk; "
               "%.3e walks/s\n",
               info.build_ms, info.grid[0], info.grid[1], info.grid[2], info.mean_list, r.kernel_ms,
               (double)r.hops_total / (double)iters, iters / (r.kernel_ms * 1e-3));
    if (cap) {
        printf("capacitance row of box %lld (F), %llu walks:\n", object, (unsigned long long)iters);
        for (int64_t k = 0; k < r.n_entries && k < r.capacity; k++)
            printf("  C[%lld,%lld] = %.6e +- %.2e\n", object, (long long)cond[k], c[k], se[k]);
    }
    if (json) {
        printf("{\"layout\": \"%s\", \"dims\": 3, \"boxes\": %lld, \"target\": %lld, \"walks\": %llu, "
               "\"seed\": %llu, \"fraction_other\": %.17g, \"escaped\": %llu, \"aborted\": %llu, "
               "\"hops_per_walk\": %.6f, \"walk_kernel_ms\": %.4f, \"walks_per_s\": %.6g, \"shell\": %.17g, "
               "\"rows\": [",
               path.c_str(), (long long)info.n, object, (unsigned long long)iters, seed, r.fraction_other,
               (unsigned long long)r.escaped, (unsigned long long)r.aborted, (double)r.hops_total / (double)iters,
               r.kernel_ms, iters / (r.kernel_ms * 1e-3), r.shell);
        for (int64_t k = 0; k < r.n_entries && k < r.capacity; k++)
            printf("%s{\"conductor\": %lld, \"hits\": %llu, \"cap\": %.17g, \"cap_se\": %.6g}", k ? ", " : "",
                   (long long)cond[k], (unsigned long long)hits[k], c[k], se[k]);
        printf("]}\n");
    }
    frw3_layout_destroy(L);
    return 0;
}

int main(int argc, char **argv) {
    std::string path = "../tests/test", hist, zspec;
    long long iters = 1000, object = 10;
    int layer = 0, device = 0;
    bool measure = false, uniform = false, cap = false, exact = false, json = false;
    unsigned long long seed = (unsigned long long)time(nullptr);
    double offset = -1.0, scale = 1.5;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto val = [&](const char *what) -> const char * {
            if (i + 1 >= argc) {
                fprintf(stderr, "%s needs a value\n", what);
                exit(2);
            }
            return argv[++i];
        };
        if (a == "-S" || a == "--source") path = val("-S");
        else if (a == "-I" || a == "--iterations") iters = atoll(val("-I"));
        else if (a == "-O" || a == "--object") object = atoll(val("-O"));
        else if (a == "-L" || a == "--layer") layer = atoi(val("-L"));
        else if (a == "-G" || a == "--GPU") {
        } else if (a == "-M" || a == "--measure") measure = true;
        else if (a == "--seed") seed = strtoull(val("--seed"), nullptr, 0);
        else if (a == "--device") device = atoi(val("--device"));
        else if (a == "--uniform") uniform = true;
        else if (a == "--offset") offset = atof(val("--offset"));
        else if (a == "--scale") scale = atof(val("--scale"));
        else if (a == "--exact-perimeter") exact = true;
        else if (a == "--cap") cap = true;
        else if (a == "--hist") hist = val("--hist");
        else if (a == "--json") json = true;
        else if (a == "--3d") zspec = val("--3d");
        else if (a == "--help" || a == "-h") {
            printf("%s", kHelp);
            return 0;
        } else {
            fprintf(stderr, "unknown argument %s\n%s", a.c_str(), kHelp);
            return 2;
        }
    }
    if (iters <= 0) {
        fprintf(stderr, "Incorrect args!\n");
        return 2;
    }
    if (!zspec.empty())
        return run3d(path, zspec, iters, object, device, seed, offset, measure, cap, json, hist);
    auto t0 = std::chrono::steady_clock::now();
    frw_layout *L = nullptr;
    if (frw_layout_from_file(path.c_str(), layer, device, &L) != FRW_OK) {
        fprintf(stderr, "error: %s\n", frw_last_error());
        return 1;
    }
    frw_layout_info info;
    frw_layout_info_get(L, &info);
    if (object < 0 || object >= info.n_rects) {
        fprintf(stderr, "Incorrect args! (object %lld of %lld rects)\n", object, (long long)info.n_rects);
        frw_layout_destroy(L);
        return 2;
    }
    frw_opts o;
    frw_opts_default(&o);
    if (offset >= 0) {
        o.gauss_mode = FRW_GAUSS_OFFSET;
        o.gauss_param = offset;
    } else {
        o.gauss_param = scale;
    }
    o.start_mode = uniform ? FRW_START_UNIFORM : FRW_START_GREEN;
    o.exact_perimeter = exact ? 1 : 0;
    std::vector<int64_t> cond(info.n_rects);
    std::vector<uint64_t> hits(info.n_rects);
    std::vector<double> c(info.n_rects), se(info.n_rects);
    frw_result r{};
    r.capacity = info.n_rects;
    r.conductor = cond.data();
    r.hits = hits.data();
    r.cap = c.data();
    r.cap_se = se.data();
    if (frw_walk(L, object, (uint64_t)iters, seed, &o, &r, nullptr) != FRW_OK) {
        fprintf(stderr, "error: %s\n", frw_last_error());
        frw_layout_destroy(L);
        return 1;
    }
    auto t1 = std::chrono::steady_clock::now();
    if (hist.empty()) hist = std::to_string((unsigned long)time(nullptr)) + "wyniki.txt";
    FILE *f = fopen(hist.c_str(), "w");
    if (f) {
        fprintf(f, "[GPU]\n");
        if (r.escaped)
            fprintf(f, "Ile scie\xc5\xbc" "ek wysz\xc5\x82o poza granice warstwy: %g%%\n",
                    (float)r.escaped / (float)iters * 100);
        std::vector<double> q(4 * info.n_rects);
        frw_layout_rects(L, q.data());
        for (int64_t k = 0; k < r.n_entries && k < r.capacity; k++)
            fprintf(f, "%g %g %g %g: %g%%\n", q[4 * cond[k]], q[4 * cond[k] + 1], q[4 * cond[k] + 2],
                    q[4 * cond[k] + 3], ((float)hits[k] / (float)iters) * 100);
        fclose(f);
        printf("Wynik zapisany do %s\n", hist.c_str());
    }
    printf("[GPU] Ile sciezek trafi\xc5\x82o do innego elementu: %f%%\n", r.fraction_other * 100.);
    printf("Czas wykonania: %lld ms\n",
           (long long)std::chrono::duration_cast<std::chrono::milliseconds>(t1 - t0).count());
    if (measure)
        printf("tree build %.3f ms (%lld nodes, depth %d); walk kernel %.3f ms; %.1f hops/walk; "
               "%.3e walks/s\n",
               info.build_ms, (long long)info.n_nodes, info.depth, r.kernel_ms,
               (double)r.hops_total / (double)iters, iters / (r.kernel_ms * 1e-3));
    if (cap && uniform) {
        printf("capacitance row of conductor %lld (F/m), %llu walks:\n", object, (unsigned long long)iters);
        for (int64_t k = 0; k < r.n_entries && k < r.capacity; k++)
            printf("  C[%lld,%lld] = %.6e +- %.2e\n", object, (long long)cond[k], c[k], se[k]);
    }
    if (json) {
        printf("{\"layout\": \"%s\", \"layer\": %d, \"rects\": %lld, \"target\": %lld, \"walks\": %llu, "
               "\"seed\": %llu, \"fraction_other\": %.17g, \"escaped\": %llu, \"aborted\": %llu, "
               "\"hops_per_walk\": %.6f, \"walk_kernel_ms\": %.4f, \"walks_per_s\": %.6g, "
               "\"tree_build_ms\": %.4f, \"gauss\": [%.17g, %.17g, %.17g, %.17g], \"rows\": [",
               path.c_str(), layer, (long long)info.n_rects, object, (unsigned long long)iters, seed, r.fraction_other,
               (unsigned long long)r.escaped, (unsigned long long)r.aborted, (double)r.hops_total / (double)iters,
               r.kernel_ms, iters / (r.kernel_ms * 1e-3), info.build_ms, r.gauss[0], r.gauss[1], r.gauss[2],
               r.gauss[3]);
        for (int64_t k = 0; k < r.n_entries && k < r.capacity; k++)
            printf("%s{\"conductor\": %lld, \"hits\": %llu, \"cap\": %.17g, \"cap_se\": %.6g}", k ? ", " : "",
                   (long long)cond[k], (unsigned long long)hits[k], c[k], se[k]);
        printf("]}\n");
    }
    frw_layout_destroy(L);
    return 0;
}
