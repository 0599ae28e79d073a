// Stand-in for a cereal header (serialization library, not in the reference tree) in
// the builds of the reference here: its build path never (de)serialises, so archives are
// declared with no-op operators.  Test and baseline infrastructure only.
#pragma once

#include <istream>
#include <ostream>

namespace cereal {
class BinaryInputArchive {
public:
    explicit BinaryInputArchive(std::istream&) {}
    template <typename... T> void operator()(T&&...) {}
};
class BinaryOutputArchive {
public:
    explicit BinaryOutputArchive(std::ostream&) {}
    template <typename... T> void operator()(T&&...) {}
};
}  // namespace cereal
