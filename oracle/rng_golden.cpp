// Known-answer generator for the oracle's restatement of the reference's
// initial-block RNG (src/core/Executor.cpp:20-62): std::mt19937(seed) feeding
// std::uniform_real_distribution<double>(-1, 1), built with the same C++
// standard library (libstdc++) as the reference. Test infrastructure only.
// Usage: rng_golden <seed> <count>  -> one %.17g value per line.
#include <cstdio>
#include <cstdlib>
#include <random>

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s seed count\n", argv[0]);
    return 2;
  }
  const unsigned seed = static_cast<unsigned>(std::strtoul(argv[1], nullptr, 10));
  const long count = std::strtol(argv[2], nullptr, 10);
  std::mt19937 rng(seed);
  std::uniform_real_distribution<double> dist(-1.0, 1.0);
  for (long i = 0; i < count; ++i) std::printf("%.17g\n", dist(rng));
  return 0;
}
