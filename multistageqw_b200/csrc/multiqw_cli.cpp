// MultiQW — drop-in replacement of the reference command
//   MultiQW n m filename [start problems]            (MultiQW.cpp:241-262)
// Same arguments (start/problems are honoured only when both are given; the
// default is 2000 problems from instance 0), same stdout ("total_t P" per
// problem) and the same output file: one float32 per problem appended to
// ./output_<n>_<m>. Differences, all reported instead of silently ignored:
// a short or missing instance file, or n/m out of range, print a message to
// stderr and exit with status 1 (the reference repeats the last instance or
// overflows). The GPU is chosen with MQW_DEVICE (default 0).
#include <cstdio>
#include <cstdlib>

#include "../../include/mqw.h"

int main(int argc, char* argv[]) {
  if (argc < 4) return -1;  // MultiQW.cpp:244
  const int n = atoi(argv[1]);
  const int m = atoi(argv[2]);
  const char* filename = argv[3];
  long long start = 0, problems = 2000;  // MultiQW.cpp:251-252
  if (argc == 6) {
    start = atoll(argv[4]);
    problems = atoll(argv[5]);
  }
  const char* dev_env = getenv("MQW_DEVICE");
  const int device = dev_env ? atoi(dev_env) : 0;
  mqw_ctx* ctx = nullptr;
  mqw_status s = mqw_create(&ctx, device);
  if (s != MQW_OK) {
    fprintf(stderr, "MultiQW: cannot open CUDA device %d: %s\n", device,
            mqw_status_string(s));
    return 1;
  }
  s = mqw_multiqw(ctx, n, m, filename, start, problems, nullptr, 1);
  if (s != MQW_OK) {
    fprintf(stderr, "MultiQW: %s: %s\n", mqw_status_string(s), mqw_last_error(ctx));
    mqw_destroy(ctx);
    return 1;
  }
  mqw_destroy(ctx);
  return 0;
}
