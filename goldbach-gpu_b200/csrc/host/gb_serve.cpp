// gb_serve.cpp -- serving loop (continuous batching of range and single-n
// requests).  Filled in with the serving entry points.
#include "gb_ctx.h"

extern "C" void gb_serve_shutdown(gb_ctx* ctx) { (void)ctx; }
