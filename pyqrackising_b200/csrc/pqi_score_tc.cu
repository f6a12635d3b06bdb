// placeholder, replaced by the tcgen05 path
#include "pqi_common.cuh"
namespace pqi {
pqi_status score_tc(const pqi_weights* w, const uint32_t* theta, int shots, double* qpart,
                    int* tiles_out, Workspace& ws, cudaStream_t s) {
  (void)w; (void)theta; (void)shots; (void)qpart; (void)tiles_out; (void)ws; (void)s;
  return PQI_ENOTSUP;
}
}  // namespace pqi
