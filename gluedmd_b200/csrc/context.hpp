// Per-Context kernel state: the CalcGluedForceKernel of this library
// (openmmapi/include/GluedKernels.h:23-105; behaviour of
// platforms/common/src/CommonGluedKernels.cpp:3805-5288 and
// platforms/common/src/CommonSerialization.cpp:20-411).
#pragma once

#include <cuda_runtime.h>
#include <string>
#include <vector>

#include "dev.hpp"
#include "force.hpp"

namespace glued {

// Owning device allocation.
struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
        return *this;
    }
    void release();
    ~DBuf();
    void alloc(size_t n);
    template <class T> T* as() const { return static_cast<T*>(p); }
    template <class T> void upload(const std::vector<T>& v, cudaStream_t s = 0);
};

void cudaCheck(cudaError_t e, const char* what);
int coordKind(float n, float m);

template <class T> void DBuf::upload(const std::vector<T>& v, cudaStream_t) {
    alloc(v.size() * sizeof(T));
    if (!v.empty()) cudaCheck(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
}

struct HostBias {
    BiasSpec spec;
    int index;     // addBias index (== energy slot)
    int local;     // index within its type
    BiasDev dev;   // host copy of the device record
    // owned buffers
    DBuf grid, centers, sigmas, logW, ints, dbls, hCenters, hHeights, mean, m2, sigma0;
    int numDeposited = 0;   // MetaD
    std::vector<int> subDeposited;   // PBMETAD: deposits per sub-grid
    int numKernelsCPU = 0;  // OPES: CPU mirror for the maxKernels guard (:5107-5110)
    int nSamplesCPU = 0;    // OPES adaptive: mirror of the GPU warm-up counter
    std::vector<double> sigma0Host;
    int depositIndex = 0;   // position in the device BiasDev array
};

class Context {
public:
    Context(const GluedForce& f, int numParticles, const double* masses);
    ~Context();

    void bind(cudaStream_t s, const void* posq, const int* atomIndex, long long* force, int padded);
    void atomsReordered();
    void setBox(const double box[9]);
    void setStep(long long step) { step_ = step; }
    double execute(bool includeForces, bool includeEnergy);
    void updateState(int step);
    std::vector<double> cvValues();
    double lastBias();
    std::vector<char> getBiasState();
    void setBiasState(const std::vector<char>& bytes);
    std::vector<double> opesMetrics(int opesIndex);
    std::vector<float> kernelSigmas(int opesIndex);
    std::vector<long long> multiWalkerPtrs(int biasIndex);
    void setMultiWalkerPtrs(int biasIndex, const std::vector<long long>& ptrs);
    int opesLastDecision(int opesIndex);
    std::vector<double> profilePhases(int reps);
    long long launchCount() const { return launches_; }
    // Sum precision: kernelSums = SumMode of the OPES / hill kernel sums;
    // coordBlocked = coordination A-side partials flushed every crun::BLK_STEPS steps.
    void setSumPrecision(int kernelSums, int coordBlocked);
    // Pair list of a cutoff coordination CV on the cell-list path (cvIndex = its
    // CV value index): (a, b) group indices, sorted (synchronizing).
    std::vector<int> cellPairs(int cvIndex);
    int sumMode() const { return sumMode_; }
    bool coordBlocked() const { return coordBlocked_; }

    int numCVs() const { return numCVs_; }
    int numRows() const { return numRows_; }
    double* dCV() const { return cvv_.as<double>(); }
    double* dGrad() const { return dudcv_.as<double>(); }
    const JacDev& jac() const { return J_; }

private:
    void buildPlan(const GluedForce& f);
    void setupBiases(const GluedForce& f);
    void enqueueExecute(cudaStream_t s, bool includeForces, int onlyPhase = -1);
    void enqueueCells(cudaStream_t s);
    int kernelsPerExecute(bool includeForces) const;
    void invalidateGraphs();
    void syncUploadBias(HostBias& hb);
    void requireBound() const;

    GluedForce force_;
    int numParticles_;
    std::vector<double> masses_;
    bool periodic_ = false;
    int numCVs_ = 0;
    int numRows_ = 0;
    long long step_ = 0;
    int lastUpdateStep_ = -1;
    bool cvReady_ = false;

    // bound OpenMM buffers
    cudaStream_t stream_ = 0;
    const float4* posq_ = nullptr;
    const int* atomIndex_ = nullptr;
    long long* force_buf_ = nullptr;
    int padded_ = 0;
    bool bound_ = false;

    // device state
    DBuf u2g_, box_, cvv_, dudcv_, energies_, testGrad_;
    DBuf jAtom_, jx_, jy_, jz_, jCv_;
    DBuf simple_, groupItems_, gAtoms_, gSlots_, gMass_, gRef_, gEv_, cmPairs_, cmParams_;
    int gAtomsN_ = 0, groupCached_ = 1;
    DBuf coordItems_, coordAtoms_, coordSlots_, coordSteps_, coordGB_, coordGA_, coordStepPosq_, coordAcc_, coordCnPiece_;
    DBuf coordSysPosq_, coordCellCn_;
    DBuf biasDev_, mergeFlag_, uprobPartial_, sumPart_;
    bool kernelSums_ = false;
    bool groupClustered_ = false;   // group CVs as one CTA cluster per CV
    bool groupBeside_ = false;      // group CVs beside the coordination grid
    bool simpleBeside_ = false;     // distance/angle/dihedral beside the coordination grid
    bool singleLane_ = false;   // any harmonic / MetaD / PBMETAD / EXTERNAL bias
    JacDev J_{};
    int numSimple_ = 0;
    GroupDev G_{};
    std::vector<CoordItem> coordItemsH_;
    std::vector<CoordStep> coordStepsH_;
    CoordRunDev R_{};
    int coordItemsN_ = 0, coordRows_ = 0, coordGrid_ = 0, coordKind_ = 3, coordAtomsN_ = 0;
    bool coordHi_ = true;
    // cutoff coordination items on the cell-list path (coord_cells.cu)
    DBuf cellItems_, cellBox_, cellScratch_;
    std::vector<CellItemDev> cellItemsH_;
    int cellItemsN_ = 0, cellTotalA_ = 0;   // every cutoff item
    int cellEvalN_ = 0, cellEvalA_ = 0;     // the first cellEvalN_: evaluated on the cell list
    int cellMaxB_ = 0, cellEvalMaxB_ = 0;   // largest B group (all / evaluated items)
    CellBox* cellBoxPinned_ = nullptr;
    int sumMode_ = SUM_FP64;        // OPES / hill kernel sums (SumMode)
    bool coordBlocked_ = false;     // coordination A sums flushed every crun::BLK_STEPS steps
    int nUprobPartial_ = 296;

    std::vector<HostBias> biases_;       // addBias order
    std::vector<int> evalOrder_;         // indices into biases_, device array order
    int numEnergySlots_ = 0;

    BoxDev boxHost_{};
    BoxDev* boxPinned_ = nullptr;
    double lastBox_[9];
    bool boxSet_ = false;
    double* energiesPinned_ = nullptr;

    cudaStream_t capStream_ = nullptr;
    cudaGraphExec_t graph_[2] = {nullptr, nullptr};
    bool useGraphs_ = true;
    long long launches_ = 0;
};

}  // namespace glued
