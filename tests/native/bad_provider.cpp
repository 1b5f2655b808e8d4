// A provider module with the B200 provider's file name and entry point but ABI version + 1
// (the reference's tests/bad_fftw_provider.cpp, for the B200 ABI). Test infrastructure.
#include "../../include/syclfft_b200_provider.h"

namespace {
const syclfft_b200_provider_v1 bad_provider{
    SYCLFFT_B200_PROVIDER_ABI_VERSION + 1, "bad-abi", nullptr, nullptr, nullptr, nullptr, nullptr,
};
}  // namespace

SYCLFFT_B200_EXPORT const syclfft_b200_provider_v1* syclfft_b200_get_provider_v1(void) { return &bad_provider; }
