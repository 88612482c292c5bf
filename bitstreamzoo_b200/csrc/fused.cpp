// Fused segment backend (placeholder until the generated-kernel path lands).
#include "fused.h"

namespace bsz {

struct FusedBackend::Impl {};

FusedBackend::FusedBackend(Device&, const ExecOptions&) : impl_(std::make_unique<Impl>()) {}
FusedBackend::~FusedBackend() = default;

void FusedBackend::run(std::vector<Node>&, const Segment&, int64_t, int64_t, unsigned long long*,
                       double*) {
  throw RuntimeError("fused mode is not available in this build");
}

}  // namespace bsz
