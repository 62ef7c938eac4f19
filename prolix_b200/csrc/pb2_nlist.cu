// Neighbour-list entry points (cutoff mode).
#include "pb2_common.cuh"
#include "pb2_kernels.cuh"

extern "C" int pb2_nl_build(pb2_batch *b, void *stream) {
  (void)stream;
  return b ? PB2_EINVAL : PB2_EINVAL;
}
extern "C" int pb2_nl_check(pb2_batch *b, int32_t *rebuilt, void *stream) {
  (void)stream;
  if (rebuilt) *rebuilt = 0;
  return b ? PB2_EINVAL : PB2_EINVAL;
}
extern "C" int pb2_nl_capacity(const pb2_batch *b, int32_t *capacity) {
  if (capacity) *capacity = 0;
  return b ? PB2_EINVAL : PB2_EINVAL;
}
extern "C" int pb2_nl_get(pb2_batch *b, int32_t *neighbors, void *stream) {
  (void)neighbors;
  (void)stream;
  return b ? PB2_EINVAL : PB2_EINVAL;
}
