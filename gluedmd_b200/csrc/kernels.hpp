// Host-callable launchers of the device kernels (plain C++ signatures).
#pragma once

#include <cuda_runtime.h>
#include <vector>
#include "../../include/glued_b200.h"
#include "dev.hpp"

namespace glued {

void launchInvertIndex(cudaStream_t s, const int* atomIndex, int* u2g, int n);
void launchComposeSimpleSlots(cudaStream_t s, SimpleItem* items, const int* u2g, int n);
void launchSimpleCVs(cudaStream_t s, const float4* posq, const int* u2g, const SimpleItem* items, int n,
                     const BoxDev* box, double* cvv, const JacDev& J,
                     bool late);
// maxCached: the largest atom range of a cached group CV (shared memory size).
void launchGroupCVs(cudaStream_t s, const float4* posq, const int* u2g, const GroupDev& G, const BoxDev* box,
                    double* cvv, const JacDev& J, int maxCached, bool clustered,
                    bool late);
void launchTestForce(cudaStream_t s, const float4* posq, const int* atomIndex, long long* force, int padded,
                     int numAtoms, int mode, double scale, const BoxDev* box);
// Coordination runs (coord_run.cuh). parts: bit 0 = pair runs, bit 1 = finalize
// (fixed-point sums -> Jacobian rows and CN values, accumulators cleared).
// kind: switch kind shared by every item of the launch (3: n = 6, m = 12;
// -1: other integer exponents; 0: non-integer exponents); hi: compare the upper
// pair bound (cutoff or x <= 1000) in the full-tile path.
// blocked: the A-side FP32 partials are flushed to the fixed-point sums every
// crun::BLK_STEPS steps of a tile run instead of once at its end.
void launchCoord(cudaStream_t s, const CoordRunDev& R, int numItems, int grid, int totalRows, int boxKind, int kind,
                 bool hi, const JacDev& J, double* cvv, int parts = 3, bool blocked = false);
void launchComposeSlots(cudaStream_t s, const int* atoms, const int* u2g, int* slots, int n);
// gB[s][ch], gA[s][ta] of a step list built with A tiles of ta and B chunks of ch atoms
void launchStepGathers(cudaStream_t s, const CoordStep* steps, int numSteps, int grid, const int* slots, int* gB,
                       int* gA, int ta = COORD_TA, int ch = COORD_CH);
int coordRunOccupancy(int kind, int boxKind, bool hi);
// out[s] = pair constants of step s (fixed items and boxes); runConstBytes() = sizeof(RunConst)
void launchStepConsts(cudaStream_t s, const CoordStep* steps, int numSteps, const CoordItem* items,
                      const BoxDev* sysBox, RunConst* out);
size_t runConstBytes();
// Cutoff coordination items on the cell-list path (coord_cells.cu): bin the B
// atoms, then pair terms into acc and the items' CN accumulators (before
// k_coord_finalize). kind as
// launchCoord. launchCellPairList: pass 1 bins and counts the pairs of every warp
// (CELL_SPLIT per A atom: pairCount[CELL_SPLIT * totalA]); pass 2 writes them
// at pairOffset (int pairs (a, b)).
void launchCellCoord(cudaStream_t s, const CellItemDev* items, int numItems, int totalA, int maxB, int kind,
                     const int* slots, const float4* posq, const CellBox* box, unsigned long long* acc);
void launchCellPairList(cudaStream_t s, const CellItemDev* items, int numItems, int totalA, int maxB, int kind,
                        const int* slots, const float4* posq, const CellBox* box, int* pairCount,
                        const long long* pairOffset, int* pairs, int pass);
// Once per (kernel, device, size): maximum shared-memory carveout and the
// dynamic shared-memory limit of a persistent runs kernel.
void runKernelSetup(const void* fn, size_t dynSmem);
// Host planning: steps tile-major (fills row0 / tilesA of the items, returns the
// accumulator row count); per-CTA ranges of numSteps over grid CTAs; whether the
// upper pair bound can bind.
// itemsPerSys: items of one system (sysPosq / sysBox entry), item-major.
int buildCoordSteps(std::vector<CoordItem>& items, int ra, int ch, std::vector<CoordStep>& steps, int itemsPerSys);
// CTA b of the persistent grid runs steps [begin[b], begin[b + 1]) (coordRange)
std::vector<int> balanceRanges(int numSteps, int grid);
// Run pieces of the static ranges (maximal sub-runs of one tile on one CTA): the
// piece slots of their last steps, item-contiguous in step order, and every
// item's slot range. Returns the number of pieces.
int buildCoordPieces(std::vector<CoordStep>& steps, const std::vector<int>& begin, std::vector<CoordItem>& items);
bool coordNeedsHi(const std::vector<CoordItem>& items, const double box[9], bool periodic);
// Kernel-sum biases (OPES, hill-sum MetaD) are summed by KSUM_CTAS CTAs per bias
// into sumPart[nb][KSUM_CTAS][9] first (kernelSums), then k_biases combines them.
constexpr int KSUM_CTAS = 64;
void launchBiases(cudaStream_t s, const BiasDev* biases, int nb, const double* cvv, int numCVs,
                  const double* testGrad, double* dUdCV, double* energies, double* sumPart, bool kernelSums,
                  bool singleLane, int sumMode = SUM_FP64);
void launchScatter(cudaStream_t s, const JacDev& J, const int* u2g, const double* dUdCV, long long* force,
                   int padded);
void launchMetadDeposit(cudaStream_t s, const BiasDev* b, const double* cvv, const double* energies);
void launchPbmetadDeposit(cudaStream_t s, const BiasDev* b, const double* cvv, int maxPoints);
void launchHillsDeposit(cudaStream_t s, const BiasDev* b, const double* cvv, const double* energies);
void launchOpesDeposit(cudaStream_t s, const BiasDev* b, const double* cvv, const double* energies,
                       int* mergeFlag, double* partial, int nPartial);

double measureFp32Peak();
// Hill-slice staging alone (staging_probe.cu): mean microseconds per launch of
// ctas CTAs staging equal slices of a numHills table with 16-byte cp.async and
// with bulk copies; status bit 0: a bulk-copy wait gave up.
void measureHillStaging(int numHills, int ctas, int reps, double* usCpAsync, double* usBulk, int* status);
void adForward(int dtype, cudaStream_t st, const glued_ad_spec& S, double* out, double* part, int nPart);
void adBackward(int dtype, cudaStream_t st, const glued_ad_spec& S, const double* out, const double* gE,
                long long* acc, void* gPos, void* gR0, void* gFrames, void* gH);
void coordinationNoAlloc(cudaStream_t stream, const void* posq, const int* groupA, int nA, const int* groupB, int nB,
                         double r0, double n, double m, int periodic, const double* box9, double* cnOut,
                         float* gradOut);

}  // namespace glued
