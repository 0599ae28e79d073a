// Stand-in for the reference's include/CdBG.hpp in the builds of src/Application.cpp here:
// that file includes it only for instantiations it leaves commented out.  Test and
// baseline infrastructure only.
#pragma once
