// External (chunked) execution: placeholder until the subgraph loader lands.
#include "engine.h"

namespace sme {
RunResult RunProgramExternal(const Program&, const HostGraph&, DeviceContext&, uint64_t, uint64_t, int,
                             uint64_t) {
  Fail(SME_ERR_INVALID_ARG, "EXTERNAL_GPU mode not available in this build");
}
}  // namespace sme
