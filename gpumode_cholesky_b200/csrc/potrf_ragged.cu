// Ragged batches: placeholder until the bucketed schedule lands.
#include "launch.h"

using namespace b2p;

extern "C" {

size_t b2p_potrf_ragged_workspace_size(const int32_t* n_host, int64_t count, int mode) {
  (void)n_host;
  (void)count;
  (void)mode;
  return 0;
}

int b2p_potrf_ragged(const float*, float*, const int64_t*, const int32_t*, const int64_t*,
                     const int32_t*, int64_t, int, void*, size_t, int32_t*, void*) {
  return set_error(B2P_ERR_UNSUPPORTED, "ragged batches are not built yet");
}

}  // extern "C"
