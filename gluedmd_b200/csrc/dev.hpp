// Device-side data layout of one context, shared by the host plan builder and the
// kernels. All atom indices held on the device are USER atom indices; kernels map
// them to OpenMM GPU slots through u2g (user -> slot), rebuilt on the device when
// OpenMM reorders atoms. All pointers are device pointers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace glued {

// Periodic box, reduced triclinic form (OpenMM): a = (ax,0,0), b = (bx,by,0),
// c = (cx,cy,cz). kind 0: no PBC; 1: rectangular; 2: triclinic.
struct __align__(16) BoxDev {
    float inv[3];
    float a[3], b[3], c[3];
    int kind;
    int pad[3];
};

// Jacobian table rows (the reference's SoA, CommonGluedKernels.h:95-100).
struct JacDev {
    int* atom;   // user atom
    float* gx;
    float* gy;
    float* gz;
    int* cv;
    int rows;
};

// Simple geometric CVs, one thread each: distance (2 atoms), angle (3), dihedral (4).
struct SimpleItem {
    int type;
    int cv;
    int jac0;
    int atoms[4];   // user atom indices
    int slot[4];    // their posq rows (rebuilt on reorder)
};

// CVs reduced by one CTA each. Field use per type:
//   COM distance : s0=g1Start s1=g2Start s2=g2End (into gAtoms/gMass), f0=M1 f1=M2
//   gyration     : s0=start s1=end, f0=M
//   RMSD / Kabsch: s0=start s1=end (gRef indexed 3*(row))
//   PCA          : s0=start s1=end (gRef, gEv)
//   path         : s0=start s1=end, r0=frame offset (atoms) into gRef, n=frames, f0=lambda
//   contact map  : s0=pair start s1=pair end (into cmPairs/cmParams)
struct GroupItem {
    int type;
    int cv;
    int jac0;
    int s0, s1, s2;
    int r0;
    int n;
    float f0, f1;
};

// Group items carried in the group kernels' parameter block (read from the
// constant bank instead of global memory).
constexpr int GROUP_INLINE = 8;

struct GroupDev {
    const GroupItem* items;
    int numItems;
    const int* atoms;
    const int* slots;      // posq row of every group atom (u2g of atoms), rebuilt on reorder
    const float* mass;
    const float* ref;      // xyz per atom (RMSD/PCA/Kabsch) or per frame-atom (path)
    const float* ev;       // PCA eigenvectors, xyz per atom
    const int2* cmPairs;
    const float4* cmParams;  // r0, n, m, w
    // the first GROUP_INLINE items again, inside the kernel's parameter block:
    // read from the constant bank instead of global memory
    GroupItem inl[GROUP_INLINE];
    int nInl;
};

struct RunConst;   // pair constants of a coordination step (coord_run.cuh)

// Coordination CVs: all-pairs tiles with deterministic partial sums.
struct CoordItem {
    int cv;
    int jac0;       // first Jacobian row (A atoms, then B atoms)
    int a0, nA;     // into coordAtoms
    int b0, nB;
    float r0, n, m;
    float rc2;      // squared cutoff, 0 = none (reference semantics)
    int kind;       // switch kind: 0 general (reference formula), k>0: m == 2n, n == 2k
    int tilesA;     // number of A tiles
    int splitsB;    // number of B splits
    int block0;     // first CTA of this item in the pair launch
    int partA;      // offset (float3 units) of this item's A partials: [splitsB][nA]
    int partB;      // offset of B partials: [tilesA][nB]
    int cn0;        // offset of this item's per-CTA CN partials
    int row0;       // first fixed-point accumulator row (A rows, then B rows)
    int pieceBegin, pieceEnd;   // this item's run-piece CN partials in cnPiece
    int cells;      // 1: cutoff item evaluated by the cell-list path (coord_cells.cu):
                    // no tile steps, no run pieces; its CN is summed in CoordRunDev::cellCn
};

struct CoordDev {
    const CoordItem* items;
    int numItems;
    const int* atoms;
    const int* blockItem;  // CTA -> item
    float* partA;          // float3 as 3 floats
    float* partB;
    double* cnPart;
    int bSplit;            // B atoms per split (multiple of the B chunk)
};

// Cutoff coordination through a cell list (coord_cells.cu). The box in FP64 for
// the cutoff decisions, which must equal the FP64 oracle's: a, b, c and the
// reciprocal diagonal 1/a_x, 1/b_y, 1/c_z; kind as BoxDev (0 none, 1
// rectangular, 2 triclinic).
struct CellBox {
    double a[3], b[3], c[3], inv[3];
    int kind, pad;
};

constexpr int CELL_MAX_DIM = 8;                      // cells per box dimension at most
constexpr int CELL_MAX = CELL_MAX_DIM * CELL_MAX_DIM * CELL_MAX_DIM;
constexpr int CELL_SPLIT = 3;   // warps per A atom (one per z slice of the stencil)

struct CellItemDev {
    int item;               // coordination item (accumulator rows, CN partials)
    int a0, nA, b0, nB;     // into the coordination atom slots
    int row0;               // first accumulator row (A rows, then B rows)
    unsigned long long* cn; // the item's CN accumulator (CoordRunDev::cellCn), 64-bit fixed point
    float r0, n, m;
    double rc2;             // rc * rc in FP64
    double rc;
    int* cellStart;         // [CELL_MAX + 1]: first sorted B atom of every cell
    int* sortedB;           // [nB]: B atom (0 .. nB - 1) of every sorted position
    float4* sortedPos;      // [nB]: its position
    int* grid;              // [4]: cells per dimension of the last binning, and their product
    int* cellId;            // [nB]: cell of every B atom (binning scratch)
    float4* posB;           // [nB]: its position (binning scratch)
    int* counts;            // [CELL_MAX]: atoms per cell (zero between steps)
};

// Coordination as static per-CTA runs of (A tile, B chunk) steps (coord_run.cuh).
constexpr int COORD_NW = 16;    // warps per CTA
constexpr int COORD_CH = 128;   // B atoms per chunk (default shape)
constexpr int COORD_TA = 128;   // A atoms per tile (16 warps x 8; default shape)
constexpr int COORD_TA_MAX = 128, COORD_CH_MAX = 256;   // largest shapes (step packing)
constexpr int COORD_F_FIRST = 1, COORD_F_LAST = 2;

// CoordStep::packed = valid A atoms (8 bits) | valid B atoms (9 bits) << 8 | flags << 17
__host__ __device__ inline int stepPack(int nA, int nB, int flags) { return nA | (nB << 8) | (flags << 17); }
__host__ __device__ inline int stepNA(int p) { return p & 0xff; }
__host__ __device__ inline int stepNB(int p) { return (p >> 8) & 0x1ff; }
__host__ __device__ inline int stepFlags(int p) { return p >> 17; }

// One (tile, chunk) step. 32 bytes.
struct __align__(16) CoordStep {
    int item;
    int aStart;          // index into slots of the tile's first A atom
    int bStart;          // index into slots of the chunk's first B atom
    int rowA;            // acc row of the tile's first A atom
    int rowB;            // acc row of the chunk's first B atom
    int packed;          // stepPack(nAv, nBv, flags (COORD_F_*))
    int pieceSlot;       // cnPiece slot of the run piece this step ends (static ranges), else -1
    int sys;             // system of the item (index into sysPosq / sysBox)
};

struct CoordRunDev {
    const CoordItem* items;
    const CoordStep* steps;
    int numSteps;              // CTA b of a grid of G runs steps [b N / G, (b + 1) N / G) (coordRange)
    const int* slots;          // per coordination atom: its row in posq
    // per-step gather tables, so that a step's gathers need no other load first:
    // gB[s][CH] = posq rows of the chunk's B atoms (-1 past the chunk: zero-fill);
    // gA[s][TA] = posq rows of the tile's A atoms when step s starts a tile run
    // (a tile's first chunk, or the first step of a CTA's range), -2 past the
    // tile (zero-fill), all -1 otherwise (no A gather)
    const int* gB;
    const int* gA;
    const float4* const* stepPosq;  // positions of the system of step s
    const float4* const* sysPosq;  // positions of system CoordStep::sys
    const BoxDev* sysBox;      // box of system CoordStep::sys
    unsigned long long* acc;   // [rows][3] fixed-point gradient sums
    const RunConst* stepConst;  // [numSteps] pair constants of every step, or nullptr: computed in the kernel
    double* cnPiece;           // CN partial of every run piece, item-contiguous (CoordItem::pieceBegin/End)
    unsigned long long* cellCn;  // [items]: CN of cell-list items in 64-bit fixed point (cleared by the reader)
};

// Equal static ranges of the coordination steps: CTA b of a grid of G runs
// steps [coordRange(N, G, b), coordRange(N, G, b + 1)).
__host__ __device__ inline int coordRange(int numSteps, int grid, int b) {
    return (int)(((long long)b * numSteps) / grid);
}

// Precision of the OPES / hill kernel sums (k_kernel_sums): FP64 evaluation and
// sums; FP32 Gaussians with plain FP32 sums; FP32 Gaussians with two-sum
// compensated FP32 sums.
enum SumMode { SUM_FP64 = 0, SUM_FP32 = 1, SUM_FP32C = 2 };

// Bias records, evaluated in the reference's bias-type order.
struct BiasDev {
    int type;
    int slot;       // biasEnergies slot (addBias order)
    int D;
    int cvIdx[8];
    int periodicFlag;       // harmonic periodic wrap
    // harmonic: k, s0 per dim (float, as the reference stores them)
    float hk[8], hs0[8];
    // MetaD grid / hills
    double h0, hif;         // initial height, 1/((gamma-1) kT) or 0
    double sigma[8];
    float isg2f[8];         // hills: 1 / sigma^2 in FP32 (FP32 kernel-sum modes)
    double origin[8], invSp[8], period[8];
    int npts[8], strides[8], per[8];
    double* grid;
    int total;
    int pace;
    // PBMETAD: sub-grid d is grid[goff[d] .. goff[d] + npts[d]); pbState = the
    // sub-grid energies [D] and softmax weights [D] of the last evaluation
    int goff[8];
    double* pbState;
    // hills table (METAD_HILLS): centers [maxH][D], heights [maxH]
    double* hCenters;
    double* hHeights;
    int* hCount;
    int maxHills;
    // OPES
    double* centers;        // [maxK][D]
    double* sigmas;         // [maxK][D]
    double* logW;           // [maxK]
    int* numKernels;
    int* numAllocated;
    double* sumUprob;       // "logZ" buffer of the reference (linear sum_uprob)
    double* sumWeights;     // KDNorm
    double* sumW;           // {sum_w, sum_w2}
    int* stepCount;
    int* nSamples;
    double* runMean;
    double* runM2;
    double* sigma0;
    int* lastDecision;
    double invGF, kT, cutoff2, eps, barrier, sigmaMin, gamma;
    int variant, adaptiveStride, maxKernels;
};

}  // namespace glued
