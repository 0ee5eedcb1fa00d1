// refgen.cpp -- TEST INFRASTRUCTURE ONLY.  Reproduces the reference client's
// input generator so that the "reference-style" regression cases use the same
// integer matrices as rocSOLVER's own gtests:
//   * std::mt19937 seeded with 69069 (clients/rocblascommon/clients_utility.cpp:19,
//     clients/rocblascommon/rocblas_random.hpp:16);
//   * every value is std::uniform_int_distribution<int>(1, 10)
//     (clients/rocblascommon/rocblas_random.hpp:104-109);
//   * rocblas_init(v, true) resets the seed and fills the whole host buffer in
//     memory order, batch member after batch member, padding rows included
//     (clients/rocblascommon/rocblas_vector.hpp:38-58).
// The distribution is implementation-defined by the C++ library; this is built
// with the system libstdc++, as the reference's clients are.
#include <cstddef>
#include <random>

extern "C" void refgen_fill(double* out, size_t count)
{
    std::mt19937 rng(69069);
    for(size_t i = 0; i < count; ++i)
        out[i] = (double)std::uniform_int_distribution<int>(1, 10)(rng);
}
