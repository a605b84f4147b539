// Test stub: RAII current-context guard.
#pragma once
#include "openmm/common/ComputeContext.h"
namespace OpenMM {
class ContextSelector {
public:
    explicit ContextSelector(ComputeContext& cc) : cc_(cc) { cc_.pushAsCurrent(); }
    ~ContextSelector() { cc_.popAsCurrent(); }
private:
    ComputeContext& cc_;
};
}  // namespace OpenMM
