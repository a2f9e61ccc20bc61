// frw_b200_bridge.cpp -- the reference's GPU entry point over the B200 library.
//
// A maintainer of the reference adds this file to randomWalk/Cuda/ in place
// of getAvgPathLenCUDA.cu (Cuda/getAvgPathLenCUDA.cu:50-80) and links
// -lfrw: every caller of getAvgPathLenCUDA (declared at
// Cuda/mainkernels.h:14; called by runRandomWalk, CPU/mainFunctions.cpp:
// 12-31) keeps its code and runs on the B200 path.  The file includes the
// reference's own header, so the definition below is checked against the
// reference's declaration when it compiles.
//
// Behaviour kept from the reference: the walks start on the target's scaled
// Gaussian surface from the Green CDF (frw_opts_default), the return value is
// the fraction of walks that did not end on RECT_ID (countAvg), the
// per-rect histogram goes to "<unixtime>wyniki.txt" in the working directory
// (saveOutput) and a failure ends the program with exit(0) as the
// reference's error paths do.  Differences: the seed is time(NULL) unless the
// environment variable FRW_SEED holds one (runs can then be reproduced), the
// `measure` flag has no timers behind it, and the device is not reset.
#include "mainkernels.h"

#include <stdio.h>
#include <stdlib.h>
#include <time.h>

#include <string>

#include "frw.h"

floatingPoint getAvgPathLenCUDA(char *path, int ITER_NUM, int RECT_ID, bool measure, int layerID) {
    (void)measure;
    const char *s = getenv("FRW_SEED");
    const uint64_t seed = (s && *s) ? strtoull(s, nullptr, 0) : (uint64_t)time(nullptr);
    const std::string hist = std::to_string((unsigned long)time(nullptr)) + "wyniki.txt";
    double fraction = 0.0;
    const frw_status st = frw_avg_path_len(path, ITER_NUM, RECT_ID, layerID, seed, /*device=*/0, hist.c_str(),
                                           &fraction);
    if (st != FRW_OK) {
        fprintf(stderr, "frw: %s\n", frw_last_error());
        exit(0);
    }
    printf("Wynik zapisany do %s\n", hist.c_str());
    return fraction;
}
