// reference_app.hpp -- the B200 path as a T_App of the reference's own Application.
//
// Compiled with the reference's include/ on the include path.  The reference runs a
// build as Application<MAX_K, T_App>(params).execute() (src/commands.cpp:185), which
// constructs T_App<k>(params) from its Build_Params for the k the user asked for
// (src/Application.cpp:9-18) and calls construct() (:50-56).  GPU_dBG_Contractor<k>
// has exactly that shape: explicit ctor from the reference's Build_Params
// (include/Build_Params.hpp:62-92), construct() running partition -> subgraphs ->
// collation on the GPU and writing <output prefix>.fa, as dBG_Contractor<k> does
// (src/dBG_Contractor.cpp:30-112).  A maintainer switches `cuttlefish build` over with
// one explicit instantiation beside the existing one (src/Application.cpp:72):
//
//     template class Application<cuttlefish::MAX_K, cuttlefish_b200::GPU_dBG_Contractor>;
//
// and Application<cuttlefish::MAX_K, cuttlefish_b200::GPU_dBG_Contractor> in cf_build.
#pragma once

#include "Build_Params.hpp"     // the reference's
#include "gpu_contractor.hpp"

namespace cuttlefish_b200 {

// The reference's parameters as the GPU path reads them: inputs (sequence files, list
// files and directories resolved by Seq_Input::seqs), k, the cutoff with the
// reference's defaults (Build_Params::cutoff: 2 for reads, 1 for references), the
// minimizer length, the output prefix and the working directory.
inline Build_Params params_from_reference(const ::Build_Params& r) {
    Build_Params p;
    p.is_read_graph = r.is_read_graph();
    p.is_ref_graph = !p.is_read_graph;
    p.seq_paths = r.sequence_input().seqs();
    p.k = r.k();
    p.cutoff = r.cutoff();
    p.min_len = r.min_len();
    p.thread_count = r.thread_count();
    p.output_prefix = r.output_prefix();
    p.working_dir = r.working_dir_path();
    return p;
}

template <uint16_t k>
class GPU_dBG_Contractor : public GPU_Contractor<k> {
public:
    explicit GPU_dBG_Contractor(const ::Build_Params& params) : GPU_Contractor<k>(params_from_reference(params)) {}
};

}  // namespace cuttlefish_b200
