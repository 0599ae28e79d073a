// Stand-in for the reference's include/dBG_Contractor.hpp in the drop-in test.
// src/Application.cpp keeps its own explicit instantiation
// Application<MAX_K, cuttlefish::dBG_Contractor> (:72); the real class needs parlaylib
// and cereal, which are not in this tree, so the test gives that T_App an empty body.
// Test infrastructure only.
#pragma once

#include "Build_Params.hpp"

#include <cstdint>

namespace cuttlefish {
template <uint16_t k>
class dBG_Contractor {
public:
    explicit dBG_Contractor(const Build_Params&) {}
    void construct() {}
};
}  // namespace cuttlefish
