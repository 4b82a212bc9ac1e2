/*
 * Reference build variant "ip3seq": the "ip3" I/P build (no B frames, three
 * references) encoded by one thread in raster order (EVX_ENABLE_WPP 0,
 * config.h:105) -- the single-thread CPU baseline of that configuration.
 * Force-included like ip1.h.
 */
#include "config.h"
#undef EVX_ENABLE_B_FRAMES
#define EVX_ENABLE_B_FRAMES (0)
#undef EVX_REFERENCE_FRAME_COUNT
#define EVX_REFERENCE_FRAME_COUNT (4)
#undef EVX_ENABLE_WPP
#define EVX_ENABLE_WPP (0)
