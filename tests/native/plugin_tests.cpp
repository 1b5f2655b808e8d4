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
    if (mode == "argument-checks") {
        // argument errors of the B200 extensions come before provider and device work
        int failures = 0;
        auto expect_invalid = [&](const char* what, auto&& fn) {
            try {
                fn();
                std::cerr << what << ": accepted\n";
                ++failures;
            } catch (const sf::exception& ex) {
                if (ex.code() != sf::error_code::invalid_argument) {
                    std::cerr << what << ": " << ex.what() << '\n';
                    ++failures;
                }
            }
        };
        expect_invalid("odd real length", [] { (void)sf::plan_dft_r2c_1d<float>(sf::queue{}, 7); });
        expect_invalid("in-place real plan", [] {
            sf::plan_options o;
            o.placement = sf::placement::in_place;
            (void)sf::plan_dft_c2r_1d<double>(sf::queue{}, 8, 1, o);
        });
        expect_invalid("overlapping output layout", [] {
            (void)sf::plan_many_dft<float>(sf::queue{}, {8}, 3, sf::direction::forward, sf::plan_options{},
                                           sf::data_layout{{1}, 8, {1}, 4});
        });
        expect_invalid("one stride for two axes", [] {
            (void)sf::plan_many_dft<float>(sf::queue{}, {8, 8}, 2, sf::direction::forward, sf::plan_options{},
                                           sf::data_layout{{8}, 64, {8, 1}, 64});
        });
        expect_invalid("zero stride", [] {
            (void)sf::plan_many_dft<double>(sf::queue{}, {8}, 2, sf::direction::forward, sf::plan_options{},
                                            sf::data_layout{{0}, 8, {1}, 8});
        });
        expect_invalid("in place with two layouts", [] {
            sf::plan_options o;
            o.placement = sf::placement::in_place;
            (void)sf::plan_many_dft<float>(sf::queue{}, {8}, 4, sf::direction::forward, o,
                                           sf::data_layout{{1}, 8, {4}, 1});
        });
        return failures == 0 ? 0 : 1;
    }
    std::cerr << "unknown mode\n";
    return 1;
} catch (const std::exception& ex) {
    std::cerr << "plugin test failed: " << ex.what() << '\n';
    return 1;
}
