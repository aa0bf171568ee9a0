// Test infrastructure only (oracle/_ref build).
// Stand-in for the absent dendrolib header that the reference's derivs.h
// includes.  Only the six face-direction names are needed; the reference uses
// them solely as bit positions in `bflag` (1u << OCT_DIR_*), so any consistent
// assignment reproduces its arithmetic.  This shim fixes the assignment to
// x-min, x-max, y-min, y-max, z-min, z-max = bits 0..5, which is also the bit
// layout of BssnBlockDesc.bflag in include/bssn_b200.h.
#pragma once
#define OCT_DIR_LEFT 0
#define OCT_DIR_RIGHT 1
#define OCT_DIR_DOWN 2
#define OCT_DIR_UP 3
#define OCT_DIR_BACK 4
#define OCT_DIR_FRONT 5
