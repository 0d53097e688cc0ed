/* ref_writer.c -- a command-line front end to the reference's cloud writers
 * (test infrastructure): reads a component-major float32 cloud from a file and
 * writes it with writeGaussianPly / writeSplat / writeSpz through
 * ref_write_cloud (oracle/ref_api.cpp). A separate process, because the PLY
 * writer's C++ streams can fail inside a host process with its own C++
 * runtime.
 *
 *   ref_writer PARAMS_FILE N REST SH_DEGREE FORMAT FRACTIONAL_BITS OUT_FILE */
#include <stdio.h>
#include <stdlib.h>

int ref_write_cloud(const float* params, int n, int rest, int cloud_sh, int format,
                    int fractional_bits, const char* path);

int main(int argc, char** argv) {
  if (argc != 8) {
    fprintf(stderr, "usage: ref_writer PARAMS N REST SH FORMAT BITS OUT\n");
    return 2;
  }
  const int n = atoi(argv[2]), rest = atoi(argv[3]);
  const size_t values = (size_t)(14 + 3 * rest) * (size_t)(n > 0 ? n : 1);
  float* params = (float*)calloc(values, sizeof(float));
  FILE* f = fopen(argv[1], "rb");
  if (params == NULL || f == NULL) return 3;
  const size_t got = fread(params, sizeof(float), values, f);
  fclose(f);
  if (n > 0 && got != values) return 4;
  const int ok = ref_write_cloud(params, n, rest, atoi(argv[4]), atoi(argv[5]), atoi(argv[6]),
                                 argv[7]);
  free(params);
  return ok ? 0 : 1;
}
