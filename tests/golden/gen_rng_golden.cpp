// Generates tests/golden/rng_golden.json from the C++ standard library that the reference's
// beam generator uses (std::mt19937_64 + std::normal_distribution, src/Beam.cpp:533-535).
// Build and run:  g++ -O2 -o /tmp/gen_rng_golden gen_rng_golden.cpp && /tmp/gen_rng_golden > rng_golden.json
#include <cstdio>
#include <random>

int main() {
    std::printf("{\n");
    const unsigned long long seeds[3] = {12345ULL, 1ULL, 987654321ULL};
    for (int s = 0; s < 3; ++s) {
        std::mt19937_64 a(seeds[s]);
        std::printf("  \"raw_%llu\": [", seeds[s]);
        for (int i = 0; i < 8; ++i) std::printf("%s\"%llu\"", i ? ", " : "", (unsigned long long)a());
        std::printf("],\n");
        std::mt19937_64 b(seeds[s]);
        std::normal_distribution<double> N01(0.0, 1.0);
        std::printf("  \"normal_%llu\": [", seeds[s]);
        for (int i = 0; i < 64; ++i) std::printf("%s%.17g", i ? ", " : "", N01(b));
        std::printf("],\n");
        std::mt19937_64 c(seeds[s]);
        std::uniform_real_distribution<double> U01(0.0, 1.0);
        std::printf("  \"uniform_%llu\": [", seeds[s]);
        for (int i = 0; i < 16; ++i) std::printf("%s%.17g", i ? ", " : "", U01(c));
        std::printf("]%s\n", s < 2 ? "," : "");
    }
    std::printf("}\n");
    return 0;
}
