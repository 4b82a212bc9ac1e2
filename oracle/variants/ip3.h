/*
 * Reference build variant "ip3": I/P-only GOP with three reference frames
 * (offsets 1 .. 3 of EVX_REFERENCE_FRAME_COUNT 4, encode.cpp:211-247).  An
 * I/P stream with exactly two references is not expressible in the reference
 * (a count of 3 breaks its log2-sized target field, serialize.cpp:233-235), so
 * this variant stands in for "2 references".  Force-included like ip1.h.
 */
#include "config.h"
#undef EVX_ENABLE_B_FRAMES
#define EVX_ENABLE_B_FRAMES (0)
#undef EVX_REFERENCE_FRAME_COUNT
#define EVX_REFERENCE_FRAME_COUNT (4)
