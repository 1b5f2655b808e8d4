// Plugin-ABI test, restating the reference's tests/plugin_tests.cpp for the B200 front
// end: with SYCLFFT_PLUGIN_PATH pointing at a module of the right file name that exports
// an incompatible ABI version (bad_provider.cpp), plan creation must fail with
// error_code::plugin_error -- before any device work, so this runs without a GPU.
// A module without the entry point must be skipped (the search moves on).
#include <cstdlib>
#include <iostream>
#include <string>

#include "../../include/syclfft_b200.hpp"

namespace sf = syclfft_b200;

int main(int argc, char** argv)
try {
    const std::string mode = argc > 1 ? argv[1] : "bad-abi";
    if (mode == "bad-abi") {
        try {
            (void)sf::plan_dft_1d<float>(sf::queue{}, 4, sf::direction::forward);
        } catch (const sf::exception& ex) {
            if (ex.code() == sf::error_code::plugin_error) return 0;
            std::cerr << "unexpected error: " << ex.what() << '\n';
            return 1;
        }
        std::cerr << "provider with incompatible ABI was accepted\n";
        return 1;
    }
    if (mode == "search-path") {
        const auto paths = sf::detail::provider_search_paths();
        // $SYCLFFT_PLUGIN_PATH entries first (empty entries dropped), then <libdir>/syclfft/providers
        if (paths.size() < 3 || paths[0] != "/first" || paths[1] != "/second") {
            std::cerr << "unexpected search path order\n";
            return 1;
        }
        if (paths.back().find("syclfft/providers") == std::string::npos) {
            std::cerr << "library-relative provider directory missing\n";
            return 1;
        }
        return 0;
    }
    if (mode == "no-symbol") {
        // the first directory holds a module without the entry point: it must be skipped;
        // the next one (the real provider) is then used, which needs a device.
        try {
            (void)sf::plan_dft_1d<float>(sf::queue{}, 4, sf::direction::forward);
            return 0;
        } catch (const sf::exception& ex) {
            if (ex.code() == sf::error_code::provider_unavailable) return 0;  // no GPU here
            std::cerr << "unexpected error: " << ex.what() << '\n';
            return 1;
        }
    }
    std::cerr << "unknown mode\n";
    return 1;
} catch (const std::exception& ex) {
    std::cerr << "plugin test failed: " << ex.what() << '\n';
    return 1;
}
