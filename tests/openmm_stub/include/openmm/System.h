// Test stub: the particle masses of OpenMM's System.
#pragma once
#include <vector>
namespace OpenMM {
class System {
public:
    int addParticle(double mass) { masses_.push_back(mass); return (int)masses_.size() - 1; }
    int getNumParticles() const { return (int)masses_.size(); }
    double getParticleMass(int index) const { return masses_[index]; }
private:
    std::vector<double> masses_;
};
}  // namespace OpenMM
