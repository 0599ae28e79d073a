// Stand-in for the reference's include/CdBG.hpp in the drop-in test: src/Application.cpp
// includes it only for instantiations it leaves commented out.  Test infrastructure only.
#pragma once
