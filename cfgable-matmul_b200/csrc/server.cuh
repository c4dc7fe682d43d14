// server.cuh -- what the rest of libcfgmm sees of the serving loop (server.cu).
#pragma once

namespace cfgmm {

// Frees the process-wide pinned staging buffers that no request holds.
void release_pinned_staging();

}  // namespace cfgmm
