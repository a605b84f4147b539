// Test stub: OpenMM's ComputeContext reorder listeners (owned and deleted by
// the context) and the current-context switch.
#pragma once
#include <vector>
namespace OpenMM {
class ComputeContext {
public:
    class ReorderListener {
    public:
        virtual ~ReorderListener() {}
        virtual void execute() = 0;
    };
    virtual ~ComputeContext() { for (ReorderListener* l : listeners_) delete l; }
    void addReorderListener(ReorderListener* listener) { listeners_.push_back(listener); }
    virtual void pushAsCurrent() {}
    virtual void popAsCurrent() {}
    // stub: what OpenMM does after it reordered the atoms
    void notifyReordered() { for (ReorderListener* l : listeners_) l->execute(); }
private:
    std::vector<ReorderListener*> listeners_;
};
}  // namespace OpenMM
