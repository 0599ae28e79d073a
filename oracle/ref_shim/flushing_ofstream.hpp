// Force-included into the build of the reference's own code here (oracle/ref_app.mk):
// every std::ofstream of the reference flushes after each write.  The reference's
// Ext_Mem_Bucket_Concurrent::close (include/Ext_Mem_Bucket.hpp) writes the last
// elements of a bucket through its std::ofstream without flushing it, and the
// discontinuity-graph expansion then reads the bucket file through a separate
// std::ifstream; a tail shorter than the stream's own buffer is not in the file yet,
// and the read fails; Unitig_Coord_Bucket_Concurrent (src/Unitig_Coord_Bucket.cpp)
// does the same.  Flushing each write changes when bytes reach the file, not which
// bytes.  Test and baseline infrastructure only.
#pragma once

#include <fstream>

namespace std {
class cf_flushing_ofstream : public basic_ofstream<char> {
public:
    using basic_ofstream<char>::basic_ofstream;
    cf_flushing_ofstream() = default;
    cf_flushing_ofstream(cf_flushing_ofstream&& o) : basic_ofstream<char>(std::move(o)) {}
    cf_flushing_ofstream& operator=(cf_flushing_ofstream&& o) {
        basic_ofstream<char>::operator=(std::move(o));
        return *this;
    }
    cf_flushing_ofstream& write(const char* s, streamsize n) {
        basic_ofstream<char>::write(s, n);
        basic_ofstream<char>::flush();
        return *this;
    }
};
}  // namespace std

#define ofstream cf_flushing_ofstream
