// Stand-in for rapidgzip's header (not in the reference tree), for building the
// reference's RabbitFX reader here: only the ISA-L configuration (USE_IGZIP, left off)
// uses rapidgzip.  Test and baseline infrastructure only.
#pragma once
