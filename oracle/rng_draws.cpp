// Random draws for the refiner oracle (test infrastructure).
//
// The reference refiner (src/refiner.cpp:46-54, src/refiner_avx2.cpp) seeds one std::mt19937
// with 12345 and, per refine iteration, draws from a fresh std::uniform_int_distribution<int>
// over [-r, r].  The mapping from engine output to distribution value is defined by the C++
// standard library in use, so it is not restated here: these helpers call the library itself.
#include <cstdint>
#include <random>

extern "C" {

void* orc_rng_create(uint32_t seed) { return new std::mt19937(seed); }

void orc_rng_destroy(void* rng) { delete static_cast<std::mt19937*>(rng); }

void orc_rng_draws(void* rng, int radius, int n, int* out) {
    auto& eng = *static_cast<std::mt19937*>(rng);
    std::uniform_int_distribution<int> dist(-radius, radius);
    for (int i = 0; i < n; ++i) out[i] = dist(eng);
}

}  // extern "C"
