// layout_io.h -- host-side layout reader, bounds rule, generator and writer.
#pragma once

#include <stdint.h>

#include <vector>

#include "../../include/frw.h"

namespace frw {
frw_status parse_layout_file(const char *path, int layer, std::vector<double> *rects, int *nlayers);
void reference_bounds(const double *rects, int64_t n, double out[4]);
void bounds_from_extent(double lx, double ty, double rx, double by, double out[4]);
frw_status generate_layout(uint64_t seed, int64_t n, double domain, int wmin, int wmax, double gap,
                           float *out);
frw_status generate_layout3(uint64_t seed, int64_t n, double domain, double zdomain, int wmin, int wmax, int zmin,
                            int zmax, double gap, float *out);
frw_status write_layout(const char *path, const float *rects, int64_t n, const char *name);
}  // namespace frw
