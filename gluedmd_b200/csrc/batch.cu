// Batched multi-walker path (placeholder until the persistent kernel lands).
#include "batch.hpp"

namespace glued {

struct Batch::Impl {};

Batch::Batch(const GluedForce&, int, const glued_walker_desc*, const double*) : impl_(nullptr) {
    throw Error(GLUED_E_UNSUPPORTED, "batched walkers are not built yet");
}
Batch::~Batch() { delete impl_; }
void Batch::setStream(cudaStream_t) {}
int Batch::autotune() { return 0; }
void Batch::execute() {}
void Batch::updateState(int) {}
void Batch::energies(double*) {}
void Batch::cvValues(double*) {}
int Batch::numHills() { return 0; }
void Batch::setHills(const double*, const double*, int) {}
int Batch::status() { return 0; }

}  // namespace glued
