// The reference's own Application<MAX_K, T_App> (src/Application.cpp, compiled where
// it lies) running the B200 path as its T_App: the reference's Build_Params is
// constructed as cf_build constructs it (src/commands.cpp:160-185), Application picks
// GPU_dBG_Contractor<k> for the requested k and execute() runs its construct(),
// which writes <output>.fa.  Test infrastructure: built by tests/dropin/Makefile.
//
//     app_dropin <k> <read|ref> <output prefix> <input file>...
#include "Application.cpp"      // the reference's src/
#include "reference_app.hpp"

#include <exception>
#include <iostream>
#include <optional>
#include <string>
#include <vector>

template class Application<cuttlefish::MAX_K, cuttlefish_b200::GPU_dBG_Contractor>;

int main(int argc, char** argv) {
    if (argc < 5) {
        std::cerr << "usage: app_dropin <k> <read|ref> <output prefix> <input file>...\n";
        return 2;
    }
    const uint16_t k = (uint16_t)std::stoi(argv[1]);
    const bool read = std::string(argv[2]) == "read";
    const std::vector<std::string> seqs(argv + 4, argv + argc);
    namespace def = cuttlefish::_default;
    const Build_Params params(read, !read, seqs, std::nullopt, std::nullopt, k, std::nullopt, false,
                              def::SUBGRAPH_COUNT, def::VERTEX_PART_COUNT, def::LMTIG_BUCKET_COUNT,
                              def::GMTIG_BUCKET_COUNT, "", "", 1, std::nullopt, false, false, def::MIN_LEN,
                              argv[3], cuttlefish::Output_Format::fa, false, false, def::WORK_DIR, false, false,
                              false, false);
    try {
        const Application<cuttlefish::MAX_K, cuttlefish_b200::GPU_dBG_Contractor> app(params);
        app.execute();
    } catch (const cuttlefish_b200::cfg_error& e) {
        std::cerr << "GPU_dBG_Contractor<" << k << ">::construct: " << e.what() << "\n";
        return 3;
    }
    return 0;
}
