/* ref_writer.c -- a command-line front end to the reference's cloud writers
 * and PLY reader (test infrastructure). A separate process, because the PLY
 * code's C++ streams can fail inside a host process with its own C++ runtime.
 *
 *   ref_writer PARAMS_FILE N REST SH_DEGREE FORMAT FRACTIONAL_BITS OUT_FILE
 *       reads a component-major float32 cloud from PARAMS_FILE and writes it
 *       with writeGaussianPly / writeSplat / writeSpz (ref_write_cloud in
 *       oracle/ref_api.cpp);
 *   ref_writer --read PLY_FILE
 *       reads it with readGaussianPly and prints "count valid min_opacity
 *       reason" (ref_read_ply_stats). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

int ref_write_cloud(const float* params, int n, int rest, int cloud_sh, int format,
                    int fractional_bits, const char* path);
int ref_read_ply_stats(const char* path, int* count, int* valid, float* min_opacity,
                       char* reason, int reason_len);

int main(int argc, char** argv) {
  if (argc == 3 && strcmp(argv[1], "--read") == 0) {
    int count = 0, valid = 0;
    float least = 0.f;
    char reason[256] = {0};
    if (!ref_read_ply_stats(argv[2], &count, &valid, &least, reason, (int)sizeof(reason))) {
      fprintf(stderr, "unreadable: %s\n", reason);
      return 1;
    }
    printf("%d %d %.9g %s\n", count, valid, least, reason[0] ? reason : "-");
    return 0;
  }
  if (argc != 8) {
    fprintf(stderr, "usage: ref_writer PARAMS N REST SH FORMAT BITS OUT | --read PLY\n");
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
