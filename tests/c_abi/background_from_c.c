/* A plain C caller of the library's host entry discoeb_background (no Python, no torch): computes
 * the background of the cosmology given on the command line (H0 Omegab Omegam mnu w0 wa) with its
 * derivative along H0, and prints the scalars of both buffers, one per line. */
#include <stdio.h>
#include <stdlib.h>

#include "discoeb.h"

int main(int argc, char** argv)
{
    if (argc != 7) return 2;
    DiscoebCosmoParams p = {atof(argv[1]), atof(argv[2]), atof(argv[3]), atof(argv[4]), atof(argv[5]), atof(argv[6]),
                            2.7255, 0.248, 2.046, 1.0, 1.0, 0.0};
    DiscoebCosmoParams dp = {1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const int N = 256;
    const int64_t size = discoeb_background_size(N);
    if (size <= 0) return 3;
    double* out = (double*)malloc(sizeof(double) * (size_t)size);
    double* out_dot = (double*)malloc(sizeof(double) * (size_t)size);
    const int32_t rc = discoeb_background(&p, &dp, 1, N, out, out_dot, 1);
    if (rc != DISCOEB_SUCCESS) return 4;
    for (int i = 0; i < DISCOEB_BGS_COUNT; ++i) printf("%.17g %.17g\n", out[i], out_dot[i]);
    free(out);
    free(out_dot);
    return 0;
}
