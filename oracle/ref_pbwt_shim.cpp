// ref_pbwt_shim.cpp — TEST INFRASTRUCTURE.
//
// Exposes the reference's own CPU PBWT builder (tcBio/SwiftImpute
// src/pbwt/pbwt_index.cpp:12-18 -> :95-151 -> :210-247) through a plain C
// symbol, so the tests can pin the oracle's restatement against the reference
// compiled from its unmodified sources. Built by oracle/Makefile into
// oracle/_ref/ (git-ignored). Nothing in the product links this.
#include "pbwt/pbwt_index.hpp"

#include <cstring>

extern "C" int ref_pbwt_build(const uint8_t* panel, uint32_t M, uint32_t N,
                              uint32_t* prefix, uint32_t* divergence) {
    try {
        swiftimpute::Logger::instance().set_level(swiftimpute::Logger::ERROR);
        auto index = swiftimpute::pbwt::PBWTIndex::build(panel, M, N);
        const size_t n = static_cast<size_t>(M) * N;
        if (prefix) std::memcpy(prefix, index->prefix().data.data(), n * sizeof(uint32_t));
        if (divergence) std::memcpy(divergence, index->divergence().data.data(), n * sizeof(uint32_t));
        return 0;
    } catch (...) {
        return 1;
    }
}
