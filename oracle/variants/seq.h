/*
 * Reference build variant "seq": the default GOP encoded by one thread in
 * raster order (EVX_ENABLE_WPP 0, config.h:105) -- the single-thread CPU
 * baseline.  Its output equals the WPP build's byte for byte.  Force-included
 * like ip1.h.
 */
#include "config.h"
#undef EVX_ENABLE_WPP
#define EVX_ENABLE_WPP (0)
