/*
 * Reference build variant "ip1": I/P-only GOP with one reference frame.
 * Force-included (-include) ahead of every reference source by oracle/Makefile:
 * it takes the reference's own config.h (its include guard then keeps later
 * includes out) and redefines two of its compile-time switches.  No reference
 * source is copied or edited.
 *   EVX_ENABLE_B_FRAMES 0        (config.h:120) P frames search the DPB by
 *                                offset from the frame index (encode.cpp:211-247)
 *   EVX_REFERENCE_FRAME_COUNT 2  (config.h:39)  offsets 1 .. 1: one reference
 */
#include "config.h"
#undef EVX_ENABLE_B_FRAMES
#define EVX_ENABLE_B_FRAMES (0)
#undef EVX_REFERENCE_FRAME_COUNT
#define EVX_REFERENCE_FRAME_COUNT (2)
