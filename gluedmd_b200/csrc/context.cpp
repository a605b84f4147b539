// Context: plan building, device state, per-step launch sequence, deposition,
// bias-state blob and read-backs.
#include "context.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>

#include "../../include/glued_b200.h"
#include "kernels.hpp"

namespace glued {

void cudaCheck(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw Error(GLUED_E_CUDA, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

DBuf::~DBuf() { release(); }

void DBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

void DBuf::alloc(size_t n) {
    if (p) { cudaFree(p); p = nullptr; }
    bytes = n;
    if (n == 0) n = 16;
    cudaCheck(cudaMalloc(&p, n), "cudaMalloc");
    cudaCheck(cudaMemset(p, 0, n), "cudaMemset");
}


namespace {

const char* cvName(int t) {
    switch (t) {
        case CV_POSITION: return "POSITION"; case CV_DRMSD: return "DRMSD"; case CV_PLANE: return "PLANE";
        case CV_PROJECTION: return "PROJECTION"; case CV_PUCKERING: return "PUCKERING";
        case CV_DIPOLE: return "DIPOLE"; case CV_VOLUME: return "VOLUME"; case CV_CELL: return "CELL";
        case CV_SECONDARY_STRUCTURE: return "SECONDARY_STRUCTURE"; case CV_ERMSD: return "ERMSD";
        case CV_ENERGY: return "ENERGY"; case CV_EXPRESSION: return "EXPRESSION"; case CV_PYTORCH: return "PYTORCH";
        default: return "?";
    }
}

bool inScopeCV(int t) {
    switch (t) {
        case CV_DISTANCE: case CV_ANGLE: case CV_DIHEDRAL: case CV_COM_DISTANCE: case CV_GYRATION:
        case CV_COORDINATION: case CV_RMSD: case CV_PATH: case CV_CONTACTMAP: case CV_PCA:
        case CV_COORDINATION_CUTOFF: case CV_RMSD_KABSCH:
            return true;
        default: return false;
    }
}

// Jacobian kind order (CommonGluedKernels.cpp:4186-4230); the two extension
// kinds follow their reference sibling.
const int kKindOrder[] = {CV_DISTANCE, CV_ANGLE, CV_DIHEDRAL, CV_COM_DISTANCE, CV_GYRATION, CV_COORDINATION,
                          CV_COORDINATION_CUTOFF, CV_RMSD, CV_RMSD_KABSCH, CV_PATH, CV_CONTACTMAP, CV_PCA};

int bodyRows(const CVSpec& c) {
    switch (c.type) {
        case CV_DISTANCE: return 2;
        case CV_ANGLE: return 3;
        case CV_DIHEDRAL: return 4;
        case CV_COORDINATION: case CV_COORDINATION_CUTOFF: return (int)c.atoms.size() - 1;
        case CV_PATH: return 2 * (int)c.atoms.size();
        case CV_CONTACTMAP: return 2 * ((int)c.atoms.size() / 2);
        default: return (int)c.atoms.size();
    }
}

}  // namespace

// Switch kind of a coordination CV: 3 for n = 6, m = 12 (sqrt- and pow-free),
// -1 for other integer exponents (cancellation-free polynomial quotient),
// 0 for non-integer exponents (the reference's pow formula).
int coordKind(float n, float m) {
    bool integral = n == std::floor(n) && m == std::floor(m) && n >= 1 && m >= 1 && n <= 64 && m <= 64;
    if (integral && n == 6.0f && m == 12.0f) return 3;
    return integral ? -1 : 0;
}

namespace {

int biasEvalRank(int t) {
    // bias evaluation order of execute() (CommonGluedKernels.cpp:4955-5026)
    switch (t) {
        case BIAS_HARMONIC: return 0;
        case BIAS_OPES: return 2;
        case BIAS_METAD: return 4;
        case BIAS_PBMETAD: return 5;
        case BIAS_EXTERNAL: return 6;
        case BIAS_METAD_HILLS: return 20;
        default: return 100;
    }
}

}  // namespace

Context::Context(const GluedForce& f, int numParticles, const double* masses)
    : force_(f), numParticles_(numParticles) {
    if (numParticles < 0) throw Error(GLUED_E_INVALID, "num_particles must be >= 0");
    masses_.assign(numParticles, 1.0);
    if (masses) for (int i = 0; i < numParticles; i++) masses_[i] = masses[i];
    periodic_ = f.usesPBC;
    std::memset(lastBox_, 0, sizeof lastBox_);
    cudaCheck(cudaMallocHost(&boxPinned_, sizeof(BoxDev)), "cudaMallocHost");
    cudaCheck(cudaMallocHost(&cellBoxPinned_, sizeof(CellBox)), "cudaMallocHost");
    cudaCheck(cudaMallocHost(&energiesPinned_, sizeof(double) * 64), "cudaMallocHost");
    cudaCheck(cudaStreamCreateWithFlags(&capStream_, cudaStreamNonBlocking), "cudaStreamCreate");
    box_.alloc(sizeof(BoxDev));
    u2g_.alloc(sizeof(int) * std::max(1, numParticles));
    boxHost_ = BoxDev{};
    boxHost_.kind = 0;
    cudaCheck(cudaMemcpy(box_.p, &boxHost_, sizeof(BoxDev), cudaMemcpyHostToDevice), "box");
    if (f.numCVSpecs() > 0) {
        buildPlan(f);
        setupBiases(f);
    }
    if (!f.testBiasGradients.empty()) {
        std::vector<double> g(std::max(numCVs_, 1), 0.0);
        for (int i = 0; i < numCVs_ && i < (int)f.testBiasGradients.size(); i++) g[i] = f.testBiasGradients[i];
        testGrad_.upload(g);
    }
}

Context::~Context() {
    invalidateGraphs();
    if (capStream_) cudaStreamDestroy(capStream_);
    if (boxPinned_) cudaFreeHost(boxPinned_);
    if (cellBoxPinned_) cudaFreeHost(cellBoxPinned_);
    if (energiesPinned_) cudaFreeHost(energiesPinned_);
}

void Context::setSumPrecision(int kernelSums, int coordBlocked) {
    if (kernelSums != SUM_FP64 && kernelSums != SUM_FP32 && kernelSums != SUM_FP32C)
        throw Error(GLUED_E_INVALID, "sum precision: kernel sums must be 0 (FP64), 1 (FP32) or 2 (FP32 two-sum)");
    if (coordBlocked != 0 && coordBlocked != 1)
        throw Error(GLUED_E_INVALID, "sum precision: coordination mode must be 0 (per tile run) or 1 (blocked)");
    if (kernelSums != sumMode_ || (coordBlocked != 0) != coordBlocked_) invalidateGraphs();
    sumMode_ = kernelSums;
    coordBlocked_ = coordBlocked != 0;
}

void Context::invalidateGraphs() {
    for (auto& g : graph_) {
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }
}

// --------------------------------------------------------------------- plan
void Context::buildPlan(const GluedForce& f) {
    numCVs_ = f.numCVValues();
    const int nSpecs = f.numCVSpecs();
    // Validation pass (CommonGluedKernels.cpp:3879-3927).
    {
        std::map<int, int> kindFirst, kindCount;
        int v = 0;
        for (int i = 0; i < nSpecs; i++) {
            const CVSpec& c = f.cv(i);
            auto err = [&](const std::string& m) { throw Error(GLUED_E_INVALID, "GluedForce CV " + std::to_string(i) + ": " + m); };
            auto needA = [&](size_t n) { if (c.atoms.size() < n) err("expected >= " + std::to_string(n) + " atoms, got " + std::to_string(c.atoms.size())); };
            auto needP = [&](size_t n) { if (c.params.size() < n) err("expected >= " + std::to_string(n) + " parameters, got " + std::to_string(c.params.size())); };
            // Every entry of atoms is range-checked, including the coordination
            // group-size slot and expression inputs, as the reference does.
            for (int a : c.atoms)
                if (a < 0 || a >= numParticles_)
                    err("atom index " + std::to_string(a) + " out of range [0," + std::to_string(numParticles_) + ")");
            int nValues = 1;
            bool contig = true;
            switch (c.type) {
                case CV_DISTANCE: needA(2); break;
                case CV_ANGLE: needA(3); break;
                case CV_DIHEDRAL: needA(4); break;
                case CV_COM_DISTANCE: needA(1); needP(1); break;
                case CV_GYRATION: needA(1); break;
                case CV_COORDINATION: case CV_COORDINATION_CUTOFF:
                    needA(2); needP(c.type == CV_COORDINATION ? 3 : 4);
                    if (c.type == CV_COORDINATION_CUTOFF && c.params.size() > 4 && c.params[4] != 0.0 &&
                        c.params[4] != 1.0)
                        err("coordination cutoff: pair search params[4] must be 0 (cell list) or 1 (all pairs)");
                    if (c.type == CV_COORDINATION_CUTOFF && !(c.params[3] > 0.0))
                        err("coordination cutoff: rc must be > 0");
                    if (c.atoms[0] < 1 || c.atoms[0] >= (int)c.atoms.size())
                        err("coordination group-A size atoms[0]=" + std::to_string(c.atoms[0]) + " invalid");
                    break;
                case CV_RMSD: case CV_RMSD_KABSCH: needA(1); needP(3 * c.atoms.size()); break;
                case CV_PATH: {
                    needP(2);
                    int N = (int)c.params[1];
                    if (N < 2) err("path needs >= 2 frames");
                    if (N > 128) err("path frame count " + std::to_string(N) + " exceeds MAX_PATH_FRAMES=128");
                    needP(2 + (size_t)N * 3 * c.atoms.size());
                    nValues = 2;
                } break;
                case CV_CONTACTMAP: needA(2); needP(4 * (c.atoms.size() / 2)); break;
                case CV_PCA: needA(1); needP(6 * c.atoms.size()); break;
                case CV_EXPRESSION: case CV_PYTORCH: contig = false; break;
                default:
                    if (c.type < 1 || c.type > 23) err("unknown CV type " + std::to_string(c.type));
            }
            if (contig) {
                if (kindFirst.find(c.type) == kindFirst.end()) kindFirst[c.type] = v;
                else if (kindFirst[c.type] + kindCount[c.type] != v)
                    err("CVs of the same kind must be added contiguously (interleaving CV kinds is unsupported)");
                kindCount[c.type] += nValues;
            }
            v += nValues;
        }
        for (int i = 0; i < nSpecs; i++) {
            const CVSpec& c = f.cv(i);
            if (!inScopeCV(c.type))
                throw Error(GLUED_E_UNSUPPORTED, std::string("GluedForce CV ") + std::to_string(i) + ": type " +
                                                     std::to_string(c.type) + " (" + cvName(c.type) +
                                                     ") is outside this library's hot path (supported: distance, angle, "
                                                     "dihedral, COM distance, gyration, coordination, RMSD, path, "
                                                     "contact map, PCA)");
        }
    }
    // Value slots and Jacobian offsets per kind.
    std::vector<int> slot(nSpecs);
    {
        int v = 0;
        for (int i = 0; i < nSpecs; i++) { slot[i] = v; v += f.cv(i).type == CV_PATH ? 2 : 1; }
    }
    std::map<int, int> kindRows, kindJac0;
    for (int i = 0; i < nSpecs; i++) kindRows[f.cv(i).type] += bodyRows(f.cv(i));
    {
        int off = 0;
        for (int t : kKindOrder) { kindJac0[t] = off; off += kindRows[t]; }
        numRows_ = off;
    }
    std::vector<int> jAtom(std::max(numRows_, 1), 0), jCv(std::max(numRows_, 1), 0);
    std::map<int, int> kindCursor;  // rows used so far inside each kind
    std::vector<SimpleItem> simple;
    std::vector<GroupItem> groups;
    std::vector<int> gAtoms;
    std::vector<float> gMass, gRef, gEv;
    std::vector<int2> cmPairs;
    std::vector<float4> cmParams;
    std::vector<CoordItem> coord;
    std::vector<double> coordRc;   // cutoff of every coordination item (0: none), FP64
    std::vector<int> coordAtoms;
    // per-kind atom cursors into the shared group arrays (the reference keeps one
    // array per kind; the row offset of an atom inside its kind is what matters)
    for (int i = 0; i < nSpecs; i++) {
        const CVSpec& c = f.cv(i);
        const int t = c.type;
        const int cv = slot[i];
        const int jac0 = kindJac0[t] + kindCursor[t];
        kindCursor[t] += bodyRows(c);
        if (t == CV_DISTANCE || t == CV_ANGLE || t == CV_DIHEDRAL) {
            SimpleItem it{};
            it.type = t; it.cv = cv; it.jac0 = jac0;
            int na = t == CV_DISTANCE ? 2 : t == CV_ANGLE ? 3 : 4;
            for (int k = 0; k < na; k++) { it.atoms[k] = c.atoms[k]; jAtom[jac0 + k] = c.atoms[k]; jCv[jac0 + k] = cv; }
            simple.push_back(it);
        } else if (t == CV_COORDINATION || t == CV_COORDINATION_CUTOFF) {
            CoordItem it{};
            it.cv = cv; it.jac0 = jac0;
            it.nA = c.atoms[0];
            it.nB = (int)c.atoms.size() - 1 - it.nA;
            it.a0 = (int)coordAtoms.size();
            it.b0 = it.a0 + it.nA;
            for (size_t k = 1; k < c.atoms.size(); k++) coordAtoms.push_back(c.atoms[k]);
            it.r0 = (float)c.params[0]; it.n = (float)c.params[1]; it.m = (float)c.params[2];
            double rc = (t == CV_COORDINATION_CUTOFF) ? c.params[3] : 0.0;
            it.rc2 = (float)(rc * rc);
            // cutoff items: all-pairs tiles with the cutoff mask, or the cell list when
            // params[4] = 1 (faster once the box spans many cutoffs)
            it.cells = (t == CV_COORDINATION_CUTOFF && c.params.size() > 4 && c.params[4] == 1.0) ? 1 : 0;
            coordRc.push_back(rc);
            it.kind = coordKind(it.n, it.m);
            for (int k = 0; k < it.nA + it.nB; k++) { jAtom[jac0 + k] = c.atoms[1 + k]; jCv[jac0 + k] = cv; }
            coord.push_back(it);
        } else {
            GroupItem it{};
            it.type = t; it.cv = cv;
            if (t == CV_COM_DISTANCE || t == CV_GYRATION || t == CV_RMSD || t == CV_RMSD_KABSCH || t == CV_PCA) {
                int s0 = (int)gAtoms.size();
                it.jac0 = jac0 - s0;  // rows addressed as jac0 + j with j the global atom slot
                for (size_t k = 0; k < c.atoms.size(); k++) {
                    gAtoms.push_back(c.atoms[k]);
                    gMass.push_back((float)masses_[c.atoms[k]]);
                    jAtom[jac0 + k] = c.atoms[k]; jCv[jac0 + k] = cv;
                }
                it.s0 = s0; it.s1 = (int)gAtoms.size(); it.s2 = it.s1;
                // keep gRef/gEv indexed by the same slot
                gRef.resize(3 * gAtoms.size(), 0.0f);
                gEv.resize(3 * gAtoms.size(), 0.0f);
                if (t == CV_COM_DISTANCE) {
                    int ng1 = (int)std::lround(c.params.empty() ? 1.0 : c.params[0]);
                    it.s1 = s0 + ng1; it.s2 = (int)gAtoms.size();
                    float m1 = 0, m2 = 0;
                    for (int j = s0; j < it.s1; j++) m1 += gMass[j];
                    for (int j = it.s1; j < it.s2; j++) m2 += gMass[j];
                    it.f0 = m1; it.f1 = m2;
                } else if (t == CV_GYRATION) {
                    float m = 0;
                    for (int j = s0; j < it.s1; j++) m += gMass[j];
                    it.f0 = m;
                } else if (t == CV_RMSD || t == CV_RMSD_KABSCH) {
                    for (size_t k = 0; k < 3 * c.atoms.size(); k++) gRef[3 * s0 + k] = (float)c.params[k];
                } else {
                    size_t n3 = 3 * c.atoms.size();
                    for (size_t k = 0; k < n3; k++) { gRef[3 * s0 + k] = (float)c.params[k]; gEv[3 * s0 + k] = (float)c.params[n3 + k]; }
                    for (size_t k = 0; k < c.atoms.size(); k++) {
                        // PCA Jacobian rows are the eigenvector (constant)
                    }
                }
            } else if (t == CV_PATH) {
                int M = (int)c.atoms.size(), N = (int)c.params[1];
                int s0 = (int)gAtoms.size();
                for (int k = 0; k < M; k++) {
                    gAtoms.push_back(c.atoms[k]);
                    gMass.push_back(1.0f);
                    jAtom[jac0 + 2 * k] = c.atoms[k]; jCv[jac0 + 2 * k] = cv;
                    jAtom[jac0 + 2 * k + 1] = c.atoms[k]; jCv[jac0 + 2 * k + 1] = cv + 1;
                }
                gRef.resize(3 * gAtoms.size(), 0.0f);
                gEv.resize(3 * gAtoms.size(), 0.0f);
                // frames appended after all per-atom data: offset in atom units
                int r0 = (int)(gRef.size() / 3);
                for (int k = 0; k < 3 * N * M; k++) gRef.push_back((float)c.params[2 + k]);
                gEv.resize(gRef.size(), 0.0f);
                // later per-atom slots must stay aligned with gAtoms: pad gAtoms/gMass too
                while ((int)gAtoms.size() < (int)(gRef.size() / 3)) { gAtoms.push_back(0); gMass.push_back(0.0f); }
                it.s0 = s0; it.s1 = s0 + M; it.r0 = r0; it.n = N; it.f0 = (float)c.params[0];
                it.jac0 = jac0;
            } else if (t == CV_CONTACTMAP) {
                int np = (int)c.atoms.size() / 2;
                it.s0 = (int)cmPairs.size();
                for (int p = 0; p < np; p++) {
                    cmPairs.push_back(make_int2(c.atoms[2 * p], c.atoms[2 * p + 1]));
                    cmParams.push_back(make_float4((float)c.params[4 * p], (float)c.params[4 * p + 1],
                                                   (float)c.params[4 * p + 2], (float)c.params[4 * p + 3]));
                    jAtom[jac0 + 2 * p] = c.atoms[2 * p]; jCv[jac0 + 2 * p] = cv;
                    jAtom[jac0 + 2 * p + 1] = c.atoms[2 * p + 1]; jCv[jac0 + 2 * p + 1] = cv;
                }
                it.s1 = (int)cmPairs.size();
                it.jac0 = jac0;
            }
            groups.push_back(it);
        }
    }
    // device uploads
    cvv_.alloc(sizeof(double) * std::max(numCVs_, 1));
    dudcv_.alloc(sizeof(double) * std::max(numCVs_, 1));
    jAtom_.upload(jAtom);
    jCv_.upload(jCv);
    jx_.alloc(sizeof(float) * std::max(numRows_, 1));
    jy_.alloc(sizeof(float) * std::max(numRows_, 1));
    jz_.alloc(sizeof(float) * std::max(numRows_, 1));
    J_.atom = jAtom_.as<int>(); J_.cv = jCv_.as<int>();
    J_.gx = jx_.as<float>(); J_.gy = jy_.as<float>(); J_.gz = jz_.as<float>();
    J_.rows = numRows_;
    simple_.upload(simple);
    numSimple_ = (int)simple.size();
    groupItems_.upload(groups);
    gAtoms_.upload(gAtoms); gMass_.upload(gMass); gRef_.upload(gRef); gEv_.upload(gEv);
    cmPairs_.upload(cmPairs); cmParams_.upload(cmParams);
    G_.items = groupItems_.as<GroupItem>(); G_.numItems = (int)groups.size();
    G_.nInl = std::min((int)groups.size(), GROUP_INLINE);
    for (int k = 0; k < G_.nInl; k++) G_.inl[k] = groups[k];
    gSlots_.alloc(sizeof(int) * std::max((size_t)1, gAtoms.size()));
    gAtomsN_ = (int)gAtoms.size();
    groupCached_ = 1;
    for (const GroupItem& gi : groups) {
        if (gi.type == CV_CONTACTMAP) continue;
        const int n = (gi.type == CV_COM_DISTANCE ? gi.s2 : gi.s1) - gi.s0;
        groupCached_ = std::max(groupCached_, n);
    }
    // large COM distance / gyration / RMSD / PCA groups: one CTA cluster per CV
    groupClustered_ = !groups.empty() && groupCached_ >= 1024;
    for (const GroupItem& gi : groups)
        if (gi.type != CV_COM_DISTANCE && gi.type != CV_GYRATION && gi.type != CV_RMSD && gi.type != CV_PCA)
            groupClustered_ = false;
    G_.atoms = gAtoms_.as<int>(); G_.slots = gSlots_.as<int>();
    G_.mass = gMass_.as<float>(); G_.ref = gRef_.as<float>();
    G_.ev = gEv_.as<float>(); G_.cmPairs = cmPairs_.as<int2>(); G_.cmParams = cmParams_.as<float4>();
    // coordination: tile-major step list over a persistent grid (coord_run.cuh)
    if (!coord.empty()) {
        // one kernel instantiation per launch: items with different switch kinds
        // fall back to the most general kind present
        coordKind_ = coord[0].kind;
        for (auto& it : coord)
            if (it.kind != coordKind_) coordKind_ = (coordKind_ == 0 || it.kind == 0) ? 0 : -1;
        if (coordKind_ != 3)
            for (auto& it : coord) it.kind = coordKind_;
        coordRows_ = buildCoordSteps(coord, 8, COORD_CH, coordStepsH_, 1 << 30);
        coordItemsN_ = (int)coord.size();
        coordAtomsN_ = (int)coordAtoms.size();
        int dev = 0, sms = 0;
        cudaCheck(cudaGetDevice(&dev), "device");
        cudaCheck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attr");
        const int occ = coordRunOccupancy(coordKind_, periodic_ ? 1 : 0, true);
        coordGrid_ = sms * occ;
        // the distance/angle/dihedral kernel (up to 256 CVs) and a few single-CTA
        // group CVs run beside the coordination grid, on SMs it leaves free (one
        // coordination CTA per SM fills an SM's registers)
        const int simpleCtas = (numSimple_ + 127) / 128;
        simpleBeside_ = numSimple_ > 0 && simpleCtas <= 2 && occ == 1 && sms > 8;
        groupBeside_ = G_.numItems > 0 && G_.numItems <= 4 && !groupClustered_ && occ == 1 && sms > 8;
        const int beside = (simpleBeside_ ? simpleCtas : 0) + (groupBeside_ ? G_.numItems : 0);
        if (beside > 0) coordGrid_ = sms - beside;
        coordGrid_ = std::max(1, std::min(coordGrid_, (int)coordStepsH_.size()));
        std::vector<int> begin = balanceRanges((int)coordStepsH_.size(), coordGrid_);
        const int pieces = buildCoordPieces(coordStepsH_, begin, coord);
        coordItemsH_ = coord;
        coordItems_.upload(coord);
        coordAtoms_.upload(coordAtoms);
        coordSlots_.alloc(sizeof(int) * std::max(1, coordAtomsN_));
        coordSteps_.upload(coordStepsH_);
        const size_t nSteps = coordStepsH_.size();
        coordGB_.alloc(sizeof(int) * COORD_CH * std::max<size_t>(1, nSteps));
        coordGA_.alloc(sizeof(int) * COORD_TA * std::max<size_t>(1, nSteps));
        coordStepPosq_.alloc(sizeof(const float4*) * std::max<size_t>(1, nSteps));
        coordSysPosq_.alloc(sizeof(const float4*));
        coordAcc_.alloc(sizeof(unsigned long long) * 3 * std::max(1, coordRows_));
        coordCnPiece_.alloc(sizeof(double) * std::max(1, pieces));
        coordCellCn_.alloc(sizeof(unsigned long long) * coord.size());
        cudaCheck(cudaMemset(coordAcc_.p, 0, coordAcc_.bytes), "coord acc");
        // cell-list items: scratch carved from one allocation, 256-byte aligned pieces
        cellItemsH_.clear();
        cellTotalA_ = 0;
        size_t bytes = 0;
        auto carve = [&](size_t n) { size_t o = bytes; bytes += (n + 255) / 256 * 256; return o; };
        std::vector<std::array<size_t, 7>> offs;
        // every cutoff item gets cell-list state (its pair list); those evaluated on
        // the cell list come first (cellEvalN_ of them)
        std::vector<size_t> order;
        for (size_t i = 0; i < coord.size(); i++)
            if (coord[i].cells) order.push_back(i);
        cellEvalN_ = (int)order.size();
        cellEvalA_ = 0;
        cellMaxB_ = cellEvalMaxB_ = 0;
        for (size_t i = 0; i < coord.size(); i++)
            if (!coord[i].cells && coordRc[i] > 0.0) order.push_back(i);
        for (size_t i : order) {
            const CoordItem& it = coord[i];
            offs.push_back({carve(sizeof(int) * (CELL_MAX + 1)), carve(sizeof(int) * std::max(1, it.nB)),
                            carve(sizeof(float4) * std::max(1, it.nB)), carve(sizeof(int) * 4),
                            carve(sizeof(int) * std::max(1, it.nB)), carve(sizeof(float4) * std::max(1, it.nB)),
                            carve(sizeof(int) * CELL_MAX)});
            CellItemDev ci{};
            ci.item = (int)i; ci.a0 = it.a0; ci.nA = it.nA; ci.b0 = it.b0; ci.nB = it.nB;
            ci.row0 = it.row0;
            ci.r0 = it.r0; ci.n = it.n; ci.m = it.m;
            ci.rc = coordRc[i];
            ci.rc2 = coordRc[i] * coordRc[i];
            cellItemsH_.push_back(ci);
            cellTotalA_ += it.nA;
            cellMaxB_ = std::max(cellMaxB_, it.nB);
            if (it.cells) {
                cellEvalA_ += it.nA;
                cellEvalMaxB_ = std::max(cellEvalMaxB_, it.nB);
            }
        }
        cellItemsN_ = (int)cellItemsH_.size();
        if (cellItemsN_ > 0) {
            cellScratch_.alloc(bytes);
            char* base = static_cast<char*>(cellScratch_.p);
            for (int k = 0; k < cellItemsN_; k++) {
                cellItemsH_[k].cellStart = reinterpret_cast<int*>(base + offs[k][0]);
                cellItemsH_[k].sortedB = reinterpret_cast<int*>(base + offs[k][1]);
                cellItemsH_[k].sortedPos = reinterpret_cast<float4*>(base + offs[k][2]);
                cellItemsH_[k].grid = reinterpret_cast<int*>(base + offs[k][3]);
                cellItemsH_[k].cellId = reinterpret_cast<int*>(base + offs[k][4]);
                cellItemsH_[k].posB = reinterpret_cast<float4*>(base + offs[k][5]);
                cellItemsH_[k].counts = reinterpret_cast<int*>(base + offs[k][6]);
            }
            for (int k = 0; k < cellItemsN_; k++)
                cellItemsH_[k].cn = coordCellCn_.as<unsigned long long>() + cellItemsH_[k].item;
            cellItems_.upload(cellItemsH_);
            CellBox cb{};
            cb.kind = 0;
            cellBox_.alloc(sizeof(CellBox));
            cudaCheck(cudaMemcpy(cellBox_.p, &cb, sizeof(CellBox), cudaMemcpyHostToDevice), "cell box");
        }
        R_.items = coordItems_.as<CoordItem>();
        R_.steps = coordSteps_.as<CoordStep>();
        R_.numSteps = (int)nSteps;
        R_.gB = coordGB_.as<int>();
        R_.gA = coordGA_.as<int>();
        R_.stepPosq = coordStepPosq_.as<const float4*>();
        R_.slots = coordSlots_.as<int>();
        R_.sysPosq = coordSysPosq_.as<const float4*>();
        R_.sysBox = box_.as<BoxDev>();
        R_.acc = coordAcc_.as<unsigned long long>();
        R_.cnPiece = coordCnPiece_.as<double>();
        R_.cellCn = coordCellCn_.as<unsigned long long>();
    }
}

void Context::setupBiases(const GluedForce& f) {
    const int nb = f.numBiases();
    std::map<int, int> typeCount;
    for (int b = 0; b < nb; b++) {
        const BiasSpec& s = f.bias(b);
        if (s.type != BIAS_HARMONIC && s.type != BIAS_METAD && s.type != BIAS_OPES && s.type != BIAS_METAD_HILLS &&
            s.type != BIAS_PBMETAD && s.type != BIAS_EXTERNAL)
            throw Error(GLUED_E_UNSUPPORTED, "GluedForce bias " + std::to_string(b) + ": type " + std::to_string(s.type) +
                                                 " is outside this library's hot path (supported: HARMONIC, METAD, "
                                                 "PBMETAD, OPES, EXTERNAL, METAD_HILLS)");
        if (s.cvs.empty() || s.cvs.size() > 8)
            throw Error(GLUED_E_INVALID, "GluedForce bias " + std::to_string(b) + ": needs 1..8 CVs");
    }
    biases_.resize(nb);
    numEnergySlots_ = nb;
    energies_.alloc(sizeof(double) * std::max(nb, 1));
    for (int b = 0; b < nb; b++) {
        HostBias& hb = biases_[b];
        hb.spec = f.bias(b);
        hb.index = b;
        hb.local = typeCount[hb.spec.type]++;
        BiasDev& d = hb.dev;
        d = BiasDev{};
        const std::vector<double>& p = hb.spec.params;
        const std::vector<int>& ip = hb.spec.iparams;
        const int D = (int)hb.spec.cvs.size();
        d.type = hb.spec.type; d.slot = b; d.D = D;
        for (int k = 0; k < D; k++) d.cvIdx[k] = hb.spec.cvs[k];
        auto needP = [&](size_t n) {
            if (p.size() < n) throw Error(GLUED_E_INVALID, "GluedForce bias " + std::to_string(b) + ": expected >= " + std::to_string(n) + " parameters");
        };
        auto needI = [&](size_t n) {
            if (ip.size() < n) throw Error(GLUED_E_INVALID, "GluedForce bias " + std::to_string(b) + ": expected >= " + std::to_string(n) + " integer parameters");
        };
        if (d.type == BIAS_HARMONIC) {
            // params [k_0, s0_0, ...] stored as float (CommonBiasKernels.cpp:115-125)
            needP(2 * D);
            for (int k = 0; k < D; k++) { d.hk[k] = (float)p[2 * k]; d.hs0[k] = (float)p[2 * k + 1]; }
            d.periodicFlag = ip.empty() ? 0 : ip[0];
        } else if (d.type == BIAS_METAD) {
            // CommonBiasKernels.cpp:206-257
            needP(3 + 3 * D); needI(1 + 2 * D);
            d.h0 = p[0];
            for (int k = 0; k < D; k++) {
                d.sigma[k] = p[1 + k];
                d.isg2f[k] = (float)(1.0 / (p[1 + k] * p[1 + k]));
            }
            double gamma = p[1 + D], kT = p[2 + D];
            d.gamma = gamma; d.kT = kT;
            d.pace = ip[0];
            int total = 1;
            for (int k = 0; k < D; k++) {
                double lo = p[3 + D + k], hi = p[3 + 2 * D + k];
                int bins = ip[1 + k];
                d.per[k] = ip[1 + D + k];
                d.origin[k] = lo;
                d.invSp[k] = bins / (hi - lo);
                d.npts[k] = bins + (d.per[k] ? 0 : 1);
                if (bins < 1) throw Error(GLUED_E_INVALID, "METAD: bins must be >= 1");
            }
            if (D > 3) throw Error(GLUED_E_INVALID, "METAD grid supports at most 3 CVs (CommonGluedKernels.cpp:3589)");
            d.strides[0] = 1;
            for (int k = 1; k < D; k++) d.strides[k] = d.strides[k - 1] * d.npts[k - 1];
            total = d.strides[D - 1] * d.npts[D - 1];
            d.total = total;
            d.hif = gamma <= 1.0 ? 0.0 : 1.0 / ((gamma - 1.0) * kT);
            hb.grid.alloc(sizeof(double) * total);
            d.grid = hb.grid.as<double>();
        } else if (d.type == BIAS_PBMETAD) {
            // N 1-D sub-grids (CommonBiasKernels.cpp:298-424):
            // params [h0, gamma, kT, sigma_0, origin_0, max_0, sigma_1, ...],
            // iparams [pace, bins_0, periodic_0, bins_1, periodic_1, ...]
            needP(3 + 3 * D); needI(1 + 2 * D);
            d.h0 = p[0];
            const double gamma = p[1], kT = p[2];
            d.gamma = gamma; d.kT = kT;
            d.pace = ip[0];
            d.hif = gamma <= 1.0 ? 0.0 : 1.0 / ((gamma - 1.0) * kT);
            int total = 0;
            for (int k = 0; k < D; k++) {
                d.sigma[k] = p[3 + 3 * k];
                const double lo = p[4 + 3 * k], hi = p[5 + 3 * k];
                const int bins = ip[1 + 2 * k];
                if (bins < 1) throw Error(GLUED_E_INVALID, "PBMETAD: bins must be >= 1");
                if (!(hi > lo)) throw Error(GLUED_E_INVALID, "PBMETAD: max must exceed origin");
                d.per[k] = ip[2 + 2 * k];
                d.origin[k] = lo;
                d.invSp[k] = bins / (hi - lo);
                d.npts[k] = bins + (d.per[k] ? 0 : 1);
                d.goff[k] = total;
                total += d.npts[k];
            }
            d.total = total;
            hb.grid.alloc(sizeof(double) * total);
            d.grid = hb.grid.as<double>();
            // last sub-grid energies 0, softmax weights 1/N (CommonBiasKernels.cpp:319-323)
            std::vector<double> st(2 * D, 0.0);
            for (int k = 0; k < D; k++) st[D + k] = 1.0 / D;
            hb.dbls.upload(st);
            d.pbState = hb.dbls.as<double>();
            hb.subDeposited.assign(D, 0);
        } else if (d.type == BIAS_EXTERNAL) {
            // user grid, no deposition (CommonBiasKernels.cpp:425-488):
            // params [origin_0.., max_0.., grid values], iparams [bins_0.., periodic_0..]
            needP(2 * D); needI(2 * D);
            if (D > 3) throw Error(GLUED_E_INVALID, "EXTERNAL grid supports at most 3 CVs (CommonGluedKernels.cpp:3589)");
            for (int k = 0; k < D; k++) {
                const double lo = p[k], hi = p[D + k];
                const int bins = ip[k];
                if (bins < 1) throw Error(GLUED_E_INVALID, "EXTERNAL: bins must be >= 1");
                d.per[k] = ip[D + k];
                d.origin[k] = lo;
                d.invSp[k] = bins / (hi - lo);
                d.npts[k] = bins + (d.per[k] ? 0 : 1);
            }
            d.strides[0] = 1;
            for (int k = 1; k < D; k++) d.strides[k] = d.strides[k - 1] * d.npts[k - 1];
            d.total = d.strides[D - 1] * d.npts[D - 1];
            needP(2 * D + (size_t)d.total);
            std::vector<double> g(p.begin() + 2 * D, p.begin() + 2 * D + d.total);
            hb.grid.upload(g);
            d.grid = hb.grid.as<double>();
        } else if (d.type == BIAS_METAD_HILLS) {
            needP(3 + 3 * D); needI(2 + D);
            d.h0 = p[0];
            for (int k = 0; k < D; k++) {
                d.sigma[k] = p[1 + k];
                d.isg2f[k] = (float)(1.0 / (p[1 + k] * p[1 + k]));
            }
            double gamma = p[1 + D], kT = p[2 + D];
            d.gamma = gamma; d.kT = kT;
            d.pace = ip[0];
            d.maxHills = ip[1];
            for (int k = 0; k < D; k++) {
                d.per[k] = ip[2 + k];
                d.period[k] = d.per[k] ? (p[3 + 2 * D + k] - p[3 + D + k]) : 0.0;
            }
            d.hif = gamma <= 1.0 ? 0.0 : 1.0 / ((gamma - 1.0) * kT);
            hb.hCenters.alloc(sizeof(double) * std::max(1, d.maxHills * D));
            hb.hHeights.alloc(sizeof(double) * std::max(1, d.maxHills));
            hb.ints.alloc(sizeof(int) * 8);
            d.hCenters = hb.hCenters.as<double>(); d.hHeights = hb.hHeights.as<double>();
            d.hCount = hb.ints.as<int>();
        } else {  // OPES (CommonBiasKernels.cpp:489-588)
            needP(3 + D);
            double kT = p[0], gamma = p[1];
            hb.sigma0Host.assign(p.begin() + 2, p.begin() + 2 + D);
            d.sigmaMin = p[2 + D];
            d.variant = ip.size() > 0 ? ip[0] : 0;
            d.pace = ip.size() > 1 ? ip[1] : 500;
            d.maxKernels = ip.size() > 2 ? ip[2] : 100000;
            bool adaptive = hb.sigma0Host[0] <= 0.0;
            d.adaptiveStride = adaptive ? (ip.size() > 3 ? ip[3] : 10 * d.pace) : 0;
            d.kT = kT; d.gamma = gamma;
            if (d.variant == 1) {
                d.invGF = 1.0; d.cutoff2 = 2.0 * gamma; d.eps = 0.0; d.barrier = gamma * kT;
            } else if (d.variant == 2) {
                if (!std::isfinite(gamma) || gamma <= 1.0)
                    throw Error(GLUED_E_INVALID, "OPES_METAD_EXPLORE (variant=2) requires finite gamma > 1");
                d.invGF = gamma - 1.0; d.cutoff2 = 2.0 * gamma; d.eps = std::exp(-gamma / (gamma - 1.0));
                d.barrier = gamma * kT;
                if (!adaptive) for (auto& s : hb.sigma0Host) s *= std::sqrt(gamma);
            } else {
                d.invGF = (gamma - 1.0) / gamma;
                d.cutoff2 = 2.0 * gamma / d.invGF;
                d.eps = std::exp(-1.0 / (d.invGF * (1.0 - d.invGF)));
                d.barrier = kT / (1.0 - d.invGF);
            }
            if (D > 16) throw Error(GLUED_E_INVALID, "OPES supports at most 16 CVs (CommonGluedKernels.cpp:2638)");
            size_t K = (size_t)std::max(1, d.maxKernels);
            hb.centers.alloc(sizeof(double) * K * D);
            hb.sigmas.alloc(sizeof(double) * K * D);
            hb.logW.alloc(sizeof(double) * K);
            {
                std::vector<double> ones(K * D, 1.0);
                cudaCheck(cudaMemcpy(hb.sigmas.p, ones.data(), sizeof(double) * K * D, cudaMemcpyHostToDevice), "opes");
            }
            hb.ints.alloc(sizeof(int) * 8);   // numKernels, numAllocated, stepCount, nSamples, lastDecision
            hb.dbls.alloc(sizeof(double) * 8); // sumUprob, sumWeights, sumW[2]
            hb.mean.alloc(sizeof(double) * D);
            hb.m2.alloc(sizeof(double) * D);
            hb.sigma0.upload(hb.sigma0Host);
            int* I = hb.ints.as<int>();
            double* Dd = hb.dbls.as<double>();
            d.centers = hb.centers.as<double>(); d.sigmas = hb.sigmas.as<double>(); d.logW = hb.logW.as<double>();
            d.numKernels = I; d.numAllocated = I + 1; d.stepCount = I + 2; d.nSamples = I + 3; d.lastDecision = I + 4;
            d.sumUprob = Dd; d.sumWeights = Dd + 1; d.sumW = Dd + 2;
            d.runMean = hb.mean.as<double>(); d.runM2 = hb.m2.as<double>(); d.sigma0 = hb.sigma0.as<double>();
            // sentinels exp(-gamma) (CommonBiasKernels.cpp:547, :599)
            double init[4] = {0.0, std::exp(-gamma), std::exp(-gamma), std::exp(-2.0 * gamma)};
            cudaCheck(cudaMemcpy(Dd, init, sizeof init, cudaMemcpyHostToDevice), "opes");
            int ii[8] = {0, 0, 0, 0, -4, 0, 0, 0};
            cudaCheck(cudaMemcpy(I, ii, sizeof ii, cudaMemcpyHostToDevice), "opes");
        }
    }
    // evaluation order: stable sort by type rank
    evalOrder_.resize(nb);
    for (int b = 0; b < nb; b++) evalOrder_[b] = b;
    std::stable_sort(evalOrder_.begin(), evalOrder_.end(), [&](int x, int y) {
        return biasEvalRank(biases_[x].spec.type) < biasEvalRank(biases_[y].spec.type);
    });
    std::vector<BiasDev> arr(std::max(nb, 1));
    for (int k = 0; k < nb; k++) { arr[k] = biases_[evalOrder_[k]].dev; biases_[evalOrder_[k]].depositIndex = k; }
    biasDev_.upload(arr);
    mergeFlag_.alloc(sizeof(int) * 4);
    uprobPartial_.alloc(sizeof(double) * nUprobPartial_);
    kernelSums_ = false;
    for (auto& hb : biases_)
        if (hb.spec.type == BIAS_OPES || hb.spec.type == BIAS_METAD_HILLS) kernelSums_ = true;
    singleLane_ = false;
    for (auto& hb : biases_)
        if (hb.spec.type == BIAS_HARMONIC || hb.spec.type == BIAS_METAD || hb.spec.type == BIAS_PBMETAD ||
            hb.spec.type == BIAS_EXTERNAL)
            singleLane_ = true;
    sumPart_.alloc(sizeof(double) * (size_t)std::max(nb, 1) * KSUM_CTAS * 9);
}

void Context::syncUploadBias(HostBias& hb) {
    cudaCheck(cudaMemcpy(biasDev_.as<BiasDev>() + hb.depositIndex, &hb.dev, sizeof(BiasDev),
                         cudaMemcpyHostToDevice), "bias upload");
}

// ---------------------------------------------------------------- binding
void Context::bind(cudaStream_t s, const void* posq, const int* atomIndex, long long* force, int padded) {
    if (padded < numParticles_) throw Error(GLUED_E_INVALID, "padded_num_atoms < num_particles");
    stream_ = s;
    posq_ = static_cast<const float4*>(posq);
    atomIndex_ = atomIndex;
    force_buf_ = force;
    padded_ = padded;
    bound_ = true;
    invalidateGraphs();
    if (coordItemsN_ > 0) {
        cudaCheck(cudaMemcpy(coordSysPosq_.p, &posq_, sizeof(posq_), cudaMemcpyHostToDevice), "coordination posq");
        std::vector<const float4*> stepPosq(std::max<size_t>(1, coordStepsH_.size()), posq_);
        cudaCheck(cudaMemcpy(coordStepPosq_.p, stepPosq.data(), sizeof(const float4*) * stepPosq.size(),
                             cudaMemcpyHostToDevice), "coordination step posq");
    }
    atomsReordered();
}

void Context::atomsReordered() {
    requireBound();
    launchInvertIndex(stream_, atomIndex_, u2g_.as<int>(), numParticles_);
    launchComposeSlots(stream_, coordAtoms_.as<int>(), u2g_.as<int>(), coordSlots_.as<int>(), coordAtomsN_);
    if (coordItemsN_ > 0)
        launchStepGathers(stream_, coordSteps_.as<CoordStep>(), (int)coordStepsH_.size(), coordGrid_,
                          coordSlots_.as<int>(), coordGB_.as<int>(), coordGA_.as<int>());
    launchComposeSlots(stream_, gAtoms_.as<int>(), u2g_.as<int>(), gSlots_.as<int>(), gAtomsN_);
    launchComposeSimpleSlots(stream_, simple_.as<SimpleItem>(), u2g_.as<int>(), numSimple_);
    cudaCheck(cudaGetLastError(), "invert index");
}

void Context::requireBound() const {
    if (!bound_) throw Error(GLUED_E_STATE, "context has no bound device buffers (call glued_context_bind)");
}

void Context::setBox(const double box[9]) {
    if (boxSet_ && std::memcmp(box, lastBox_, sizeof lastBox_) == 0) return;
    std::memcpy(lastBox_, box, sizeof lastBox_);
    boxSet_ = true;
    BoxDev b{};
    for (int i = 0; i < 3; i++) { b.a[i] = (float)box[i]; b.b[i] = (float)box[3 + i]; b.c[i] = (float)box[6 + i]; }
    b.inv[0] = (float)(1.0 / box[0]); b.inv[1] = (float)(1.0 / box[4]); b.inv[2] = (float)(1.0 / box[8]);
    bool rect = box[1] == 0 && box[2] == 0 && box[3] == 0 && box[5] == 0 && box[6] == 0 && box[7] == 0;
    b.kind = periodic_ ? (rect ? 1 : 2) : 0;
    if (b.kind != boxHost_.kind) invalidateGraphs();
    boxHost_ = b;
    if (coordItemsN_ > 0) {
        bool hi = coordNeedsHi(coordItemsH_, box, periodic_);
        if (hi != coordHi_) invalidateGraphs();
        coordHi_ = hi;
    }
    // The device copy is read by graph-replayed kernels: stage through pinned memory
    // on the same stream so it is ordered before the next launch.
    if (bound_) {
        cudaCheck(cudaStreamSynchronize(stream_), "box sync");
        *boxPinned_ = b;
        cudaCheck(cudaMemcpyAsync(box_.p, boxPinned_, sizeof(BoxDev), cudaMemcpyHostToDevice, stream_), "box");
    } else {
        cudaCheck(cudaMemcpy(box_.p, &b, sizeof(BoxDev), cudaMemcpyHostToDevice), "box");
    }
    if (cellItemsN_ > 0) {
        // FP64 box of the cell-list decisions (the oracle's: 1 / diagonal in FP64)
        CellBox cb{};
        for (int i = 0; i < 3; i++) { cb.a[i] = box[i]; cb.b[i] = box[3 + i]; cb.c[i] = box[6 + i]; }
        cb.inv[0] = 1.0 / box[0]; cb.inv[1] = 1.0 / box[4]; cb.inv[2] = 1.0 / box[8];
        cb.kind = b.kind;
        if (bound_) {
            *cellBoxPinned_ = cb;
            cudaCheck(cudaMemcpyAsync(cellBox_.p, cellBoxPinned_, sizeof(CellBox), cudaMemcpyHostToDevice, stream_),
                      "cell box");
        } else {
            cudaCheck(cudaMemcpy(cellBox_.p, &cb, sizeof(CellBox), cudaMemcpyHostToDevice), "cell box");
        }
    }
}

// ---------------------------------------------------------------- execute
// Launch groups of one force evaluation, in order:
//   0 simple CVs, 1 group CVs, 2 coordination pairs, 3 coordination finalize,
//   4 biases, 5 scatter; with simpleBeside_ / groupBeside_ those CV kernels come
//   after the pairs and run on the SMs the pair grid leaves free. onlyPhase >= 0
//   enqueues a single group (profiling).
void Context::enqueueExecute(cudaStream_t s, bool includeForces, int onlyPhase) {
    const BoxDev* box = box_.as<BoxDev>();
    double* cvv = cvv_.as<double>();
    const int* u2g = u2g_.as<int>();
    auto want = [&](int p) { return onlyPhase < 0 || onlyPhase == p; };
    if ((simpleBeside_ || groupBeside_) && onlyPhase < 0) {
        // coordination pairs, the CV kernels that fit beside them, then the finalize
        if (!simpleBeside_) launchSimpleCVs(s, posq_, u2g, simple_.as<SimpleItem>(), numSimple_, box, cvv, J_, false);
        if (!groupBeside_) launchGroupCVs(s, posq_, u2g, G_, box, cvv, J_, groupCached_, groupClustered_, false);
        launchCoord(s, R_, coordItemsN_, coordGrid_, coordRows_, boxHost_.kind, coordKind_, coordHi_, J_, cvv, 1,
                    coordBlocked_);
        if (simpleBeside_) launchSimpleCVs(s, posq_, u2g, simple_.as<SimpleItem>(), numSimple_, box, cvv, J_, true);
        if (groupBeside_) launchGroupCVs(s, posq_, u2g, G_, box, cvv, J_, groupCached_, groupClustered_, true);
        enqueueCells(s);
        launchCoord(s, R_, coordItemsN_, coordGrid_, coordRows_, boxHost_.kind, coordKind_, coordHi_, J_, cvv, 2,
                    coordBlocked_);
    } else {
        if (want(0)) launchSimpleCVs(s, posq_, u2g, simple_.as<SimpleItem>(), numSimple_, box, cvv, J_, false);
        if (want(1)) launchGroupCVs(s, posq_, u2g, G_, box, cvv, J_, groupCached_, groupClustered_, false);
        if (want(2))
            launchCoord(s, R_, coordItemsN_, coordGrid_, coordRows_, boxHost_.kind, coordKind_, coordHi_, J_, cvv, 1,
                        coordBlocked_);
        if (want(2)) enqueueCells(s);
        if (want(3))
            launchCoord(s, R_, coordItemsN_, coordGrid_, coordRows_, boxHost_.kind, coordKind_, coordHi_, J_, cvv, 2,
                        coordBlocked_);
    }
    if (want(4))
        launchBiases(s, biasDev_.as<BiasDev>(), (int)biases_.size(), cvv, numCVs_,
                     testGrad_.p ? testGrad_.as<double>() : nullptr, dudcv_.as<double>(), energies_.as<double>(),
                     sumPart_.as<double>(), kernelSums_, singleLane_, sumMode_);
    if (includeForces && want(5)) launchScatter(s, J_, u2g, dudcv_.as<double>(), force_buf_, padded_);
}

void Context::enqueueCells(cudaStream_t s) {
    launchCellCoord(s, cellItems_.as<CellItemDev>(), cellEvalN_, cellEvalA_, cellEvalMaxB_, coordKind_,
                    coordSlots_.as<int>(), static_cast<const float4*>(posq_), cellBox_.as<CellBox>(),
                    coordAcc_.as<unsigned long long>());
}

std::vector<int> Context::cellPairs(int cvIndex) {
    requireBound();
    int k = -1;
    for (int i = 0; i < cellItemsN_; i++)
        if (coordItemsH_[cellItemsH_[i].item].cv == cvIndex) k = i;
    if (k < 0) throw Error(GLUED_E_INVALID, "cell pairs: CV " + std::to_string(cvIndex) +
                                                " is not a cutoff coordination");
    const int nA = cellItemsH_[k].nA;
    int a0 = 0;
    for (int i = 0; i < k; i++) a0 += cellItemsH_[i].nA;
    // one count / offset per warp: CELL_SPLIT warps per A atom
    const int nw = CELL_SPLIT * cellTotalA_;
    DBuf cnt, off, pairs;
    cnt.alloc(sizeof(int) * std::max(1, nw));
    off.alloc(sizeof(long long) * std::max(1, nw));
    launchCellPairList(stream_, cellItems_.as<CellItemDev>(), cellItemsN_, cellTotalA_, cellMaxB_, coordKind_,
                       coordSlots_.as<int>(), static_cast<const float4*>(posq_), cellBox_.as<CellBox>(), cnt.as<int>(),
                       nullptr, nullptr, 1);
    std::vector<int> c(nw);
    cudaCheck(cudaMemcpyAsync(c.data(), cnt.p, sizeof(int) * c.size(), cudaMemcpyDeviceToHost, stream_), "pairs");
    cudaCheck(cudaStreamSynchronize(stream_), "pairs");
    std::vector<long long> o(nw + 1, 0);
    for (int i = 0; i < nw; i++) o[i + 1] = o[i] + c[i];
    cudaCheck(cudaMemcpy(off.p, o.data(), sizeof(long long) * nw, cudaMemcpyHostToDevice), "pairs");
    pairs.alloc(sizeof(int) * 2 * std::max<long long>(1, o[nw]));
    launchCellPairList(stream_, cellItems_.as<CellItemDev>(), cellItemsN_, cellTotalA_, cellMaxB_, coordKind_,
                       coordSlots_.as<int>(), static_cast<const float4*>(posq_), cellBox_.as<CellBox>(), nullptr,
                       off.as<long long>(), pairs.as<int>(), 2);
    const long long p0 = o[CELL_SPLIT * a0], p1 = o[CELL_SPLIT * (a0 + nA)];
    std::vector<int> out(2 * (p1 - p0));
    if (p1 > p0)
        cudaCheck(cudaMemcpyAsync(out.data(), pairs.as<int>() + 2 * p0, sizeof(int) * out.size(),
                                  cudaMemcpyDeviceToHost, stream_), "pairs");
    cudaCheck(cudaStreamSynchronize(stream_), "pairs");
    std::vector<std::pair<int, int>> v(p1 - p0);
    for (size_t i = 0; i < v.size(); i++) v[i] = {out[2 * i], out[2 * i + 1]};
    std::sort(v.begin(), v.end());
    for (size_t i = 0; i < v.size(); i++) { out[2 * i] = v[i].first; out[2 * i + 1] = v[i].second; }
    return out;
}

int Context::kernelsPerExecute(bool includeForces) const {
    int k = 1;  // biases
    if (kernelSums_ && !testGrad_.p && !biases_.empty()) k++;
    if (numSimple_ > 0) k++;
    if (G_.numItems > 0) k++;
    if (coordItemsN_ > 0) k += (coordStepsH_.empty() ? 1 : 2) + (cellEvalN_ > 0 ? 2 : 0);
    if (includeForces && numRows_ > 0) k++;
    return k;
}

std::vector<double> Context::profilePhases(int reps) {
    requireBound();
    if (reps < 1) reps = 1;
    std::vector<double> out(6, 0.0);
    if (numCVs_ == 0) return out;
    cudaEvent_t a, b;
    cudaCheck(cudaEventCreate(&a), "event");
    cudaCheck(cudaEventCreate(&b), "event");
    for (int p = 0; p < 6; p++) {
        enqueueExecute(stream_, true, p);  // warm-up
        cudaCheck(cudaEventRecord(a, stream_), "event");
        for (int r = 0; r < reps; r++) enqueueExecute(stream_, true, p);
        cudaCheck(cudaEventRecord(b, stream_), "event");
        cudaCheck(cudaEventSynchronize(b), "event");
        float ms = 0;
        cudaCheck(cudaEventElapsedTime(&ms, a, b), "event");
        out[p] = ms / reps;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    // the pair-only repetitions left sums that no finalize cleared
    if (coordItemsN_ > 0) {
        cudaCheck(cudaMemsetAsync(coordAcc_.p, 0, coordAcc_.bytes, stream_), "coord acc");
    }
    return out;
}

double Context::execute(bool includeForces, bool includeEnergy) {
    requireBound();
    if (force_.testForceMode != 0) {
        launchTestForce(stream_, posq_, atomIndex_, force_buf_, padded_, numParticles_, force_.testForceMode,
                        force_.testForceScale, box_.as<BoxDev>());
        launches_ += 1;
        cudaCheck(cudaGetLastError(), "test force");
        return 0.0;
    }
    if (numCVs_ == 0) return 0.0;
    int gi = includeForces ? 1 : 0;
    if (useGraphs_) {
        if (!graph_[gi]) {
            cudaGraph_t g;
            cudaCheck(cudaStreamBeginCapture(capStream_, cudaStreamCaptureModeThreadLocal), "capture begin");
            enqueueExecute(capStream_, includeForces);
            cudaError_t e = cudaStreamEndCapture(capStream_, &g);
            cudaCheck(e, "capture end");
            cudaCheck(cudaGraphInstantiate(&graph_[gi], g, 0), "graph instantiate");
            cudaGraphDestroy(g);
        }
        cudaCheck(cudaGraphLaunch(graph_[gi], stream_), "graph launch");
    } else {
        enqueueExecute(stream_, includeForces);
        cudaCheck(cudaGetLastError(), "execute");
    }
    launches_ += kernelsPerExecute(includeForces);
    cvReady_ = true;
    double total = 0.0;
    if (includeEnergy && numEnergySlots_ > 0) {
        int n = std::min(numEnergySlots_, 64);
        cudaCheck(cudaMemcpyAsync(energiesPinned_, energies_.p, sizeof(double) * n, cudaMemcpyDeviceToHost, stream_),
                  "energy download");
        cudaCheck(cudaStreamSynchronize(stream_), "energy sync");
        for (int i = 0; i < n; i++) total += energiesPinned_[i];
        if (numEnergySlots_ > 64) {
            std::vector<double> rest(numEnergySlots_);
            cudaCheck(cudaMemcpy(rest.data(), energies_.p, sizeof(double) * numEnergySlots_, cudaMemcpyDeviceToHost), "energy");
            total = 0.0;
            for (double e : rest) total += e;
        }
    }
    return total;
}

// ------------------------------------------------------------ updateState
void Context::updateState(int step) {
    // CommonGluedKernels.cpp:5050-5157: deposits use the previous execute()'s
    // cvValues and bias energies; never before the first execute, once per step,
    // not at step 0, OPES before MetaD.
    step_ = step;
    if (!cvReady_) return;
    if (step == lastUpdateStep_) return;
    bool any = false;
    for (auto& hb : biases_)
        if (hb.spec.type == BIAS_OPES || hb.spec.type == BIAS_METAD || hb.spec.type == BIAS_METAD_HILLS ||
            hb.spec.type == BIAS_PBMETAD)
            any = true;
    if (!any) return;
    lastUpdateStep_ = step;
    requireBound();
    const double* cvv = cvv_.as<double>();
    const double* en = energies_.as<double>();
    for (auto& hb : biases_) {
        if (hb.spec.type != BIAS_OPES) continue;
        if (step == 0 || step % hb.dev.pace != 0) continue;
        if (hb.numKernelsCPU >= hb.dev.maxKernels) continue;
        bool will = hb.dev.adaptiveStride == 0 || hb.nSamplesCPU >= hb.dev.adaptiveStride;
        launchOpesDeposit(stream_, biasDev_.as<BiasDev>() + hb.depositIndex, cvv, en, mergeFlag_.as<int>(),
                          uprobPartial_.as<double>(), nUprobPartial_);
        launches_ += 3;
        if (will) hb.numKernelsCPU++;
    }
    for (auto& hb : biases_) {
        if (hb.spec.type == BIAS_METAD) {
            if (step == 0 || step % hb.dev.pace != 0) continue;
            launchMetadDeposit(stream_, biasDev_.as<BiasDev>() + hb.depositIndex, cvv, en);
            launches_ += 1;
            hb.numDeposited++;
        }
    }
    // PBMETAD after MetaD (CommonGluedKernels.cpp:5147-5155)
    for (auto& hb : biases_) {
        if (hb.spec.type != BIAS_PBMETAD) continue;
        if (step == 0 || step % hb.dev.pace != 0) continue;
        int maxPoints = 0;
        for (int k = 0; k < hb.dev.D; k++) maxPoints = std::max(maxPoints, hb.dev.npts[k]);
        launchPbmetadDeposit(stream_, biasDev_.as<BiasDev>() + hb.depositIndex, cvv, maxPoints);
        launches_ += 1;
        for (auto& n : hb.subDeposited) n++;
    }
    for (auto& hb : biases_) {
        if (hb.spec.type == BIAS_METAD_HILLS) {
            if (step == 0 || step % hb.dev.pace != 0) continue;
            launchHillsDeposit(stream_, biasDev_.as<BiasDev>() + hb.depositIndex, cvv, en);
            launches_ += 1;
        }
    }
    cudaCheck(cudaGetLastError(), "updateState");
}

// ---------------------------------------------------------------- reads
std::vector<double> Context::cvValues() {
    if (numCVs_ == 0) return {};
    std::vector<double> v(numCVs_);
    if (bound_) cudaCheck(cudaStreamSynchronize(stream_), "sync");
    cudaCheck(cudaMemcpy(v.data(), cvv_.p, sizeof(double) * numCVs_, cudaMemcpyDeviceToHost), "cv download");
    return v;
}

double Context::lastBias() {
    if (numEnergySlots_ == 0) return 0.0;
    std::vector<double> e(numEnergySlots_);
    if (bound_) cudaCheck(cudaStreamSynchronize(stream_), "sync");
    cudaCheck(cudaMemcpy(e.data(), energies_.p, sizeof(double) * numEnergySlots_, cudaMemcpyDeviceToHost), "bias");
    double t = 0;
    for (double x : e) t += x;
    return t;
}

// Multiwalker sharing: raw device pointers of a bias's shared arrays.
std::vector<long long> Context::multiWalkerPtrs(int biasIndex) {
    if (biasIndex < 0 || biasIndex >= (int)biases_.size()) throw Error(GLUED_E_INVALID, "GluedForce: bias index out of range");
    HostBias& hb = biases_[biasIndex];
    if (hb.spec.type == BIAS_METAD) return {(long long)(uintptr_t)hb.dev.grid};
    if (hb.spec.type == BIAS_OPES)
        return {(long long)(uintptr_t)hb.dev.centers, (long long)(uintptr_t)hb.dev.sigmas,
                (long long)(uintptr_t)hb.dev.logW, (long long)(uintptr_t)hb.dev.numKernels,
                (long long)(uintptr_t)hb.dev.numAllocated};
    return {};
}

void Context::setMultiWalkerPtrs(int biasIndex, const std::vector<long long>& ptrs) {
    if (biasIndex < 0 || biasIndex >= (int)biases_.size()) throw Error(GLUED_E_INVALID, "GluedForce: bias index out of range");
    HostBias& hb = biases_[biasIndex];
    if (hb.spec.type == BIAS_METAD) {
        if (ptrs.size() < 1) throw Error(GLUED_E_INVALID, "METAD multiwalker pointers: expected [grid]");
        hb.dev.grid = reinterpret_cast<double*>((uintptr_t)ptrs[0]);
    } else if (hb.spec.type == BIAS_OPES) {
        if (ptrs.size() < 5) throw Error(GLUED_E_INVALID, "OPES multiwalker pointers: expected 5");
        hb.dev.centers = reinterpret_cast<double*>((uintptr_t)ptrs[0]);
        hb.dev.sigmas = reinterpret_cast<double*>((uintptr_t)ptrs[1]);
        hb.dev.logW = reinterpret_cast<double*>((uintptr_t)ptrs[2]);
        hb.dev.numKernels = reinterpret_cast<int*>((uintptr_t)ptrs[3]);
        hb.dev.numAllocated = reinterpret_cast<int*>((uintptr_t)ptrs[4]);
    } else {
        return;
    }
    if (bound_) cudaCheck(cudaStreamSynchronize(stream_), "sync");
    syncUploadBias(hb);
}

int Context::opesLastDecision(int opesIndex) {
    int k = 0;
    for (auto& hb : biases_) {
        if (hb.spec.type != BIAS_OPES) continue;
        if (k++ != opesIndex) continue;
        int v = 0;
        if (bound_) cudaCheck(cudaStreamSynchronize(stream_), "sync");
        cudaCheck(cudaMemcpy(&v, hb.dev.lastDecision, sizeof(int), cudaMemcpyDeviceToHost), "decision");
        return v;
    }
    throw Error(GLUED_E_INVALID, "opes index out of range");
}

std::vector<double> Context::opesMetrics(int opesIndex) {
    // CommonGluedKernels.cpp:5164-5210
    int k = 0;
    for (auto& hb : biases_) {
        if (hb.spec.type != BIAS_OPES) continue;
        if (k++ != opesIndex) continue;
        if (bound_) cudaCheck(cudaStreamSynchronize(stream_), "sync");
        double dd[4];
        cudaCheck(cudaMemcpy(dd, hb.dev.sumUprob, sizeof(double) * 4, cudaMemcpyDeviceToHost), "metrics");
        // each counter through its own pointer: a secondary walker's numKernels
        // points into the primary's table, its deposit counter stays its own
        int nker = 0, steps = 0;
        cudaCheck(cudaMemcpy(&nker, hb.dev.numKernels, sizeof(int), cudaMemcpyDeviceToHost), "metrics");
        cudaCheck(cudaMemcpy(&steps, hb.dev.stepCount, sizeof(int), cudaMemcpyDeviceToHost), "metrics");
        double sumUp = hb.numKernelsCPU > 0 ? dd[0] : 0.0;
        double counter = (double)steps;
        double KDEnorm = hb.dev.variant == 2 ? counter : dd[1];
        double zed = (nker > 0 && KDEnorm > 0.0) ? sumUp / (KDEnorm * (double)nker) : 1.0;
        double rct = (counter > 0.0 && dd[1] > 0.0) ? hb.dev.kT * std::log(dd[1] / counter) : 0.0;
        double neff = (1.0 + dd[2]) * (1.0 + dd[2]) / (1.0 + dd[3]);
        return {zed, rct, (double)nker, neff};
    }
    throw Error(GLUED_E_INVALID, "getOPESMetrics: biasIndex out of range");
}

std::vector<float> Context::kernelSigmas(int opesIndex) {
    int k = 0;
    for (auto& hb : biases_) {
        if (hb.spec.type != BIAS_OPES) continue;
        if (k++ != opesIndex) continue;
        if (bound_) cudaCheck(cudaStreamSynchronize(stream_), "sync");
        int nk = 0;
        cudaCheck(cudaMemcpy(&nk, hb.dev.numKernels, sizeof(int), cudaMemcpyDeviceToHost), "sigmas");
        if (nk <= 0) return {};
        std::vector<double> s((size_t)nk * hb.dev.D);
        cudaCheck(cudaMemcpy(s.data(), hb.dev.sigmas, sizeof(double) * s.size(), cudaMemcpyDeviceToHost), "sigmas");
        return std::vector<float>(s.begin(), s.end());
    }
    return {};
}

// ------------------------------------------------------- bias-state blob
// 'GPUS' v1 layout of platforms/common/src/CommonSerialization.cpp:20-177. OPES,
// METAD and PBMETAD carry state in this library; EXTERNAL is written as its count
// only (its grid is fixed at construction); the counts of the other reference
// sections are written as 0 so a reference reader accepts the blob. State of the
// hill-sum extension follows the reference sections under its own 'HILL' tag,
// which a reference reader ignores (it stops after its last section).
std::vector<char> Context::getBiasState() {
    if (bound_) cudaCheck(cudaStreamSynchronize(stream_), "sync");
    std::vector<char> buf;
    auto w = [&](const void* src, size_t n) { const char* p = (const char*)src; buf.insert(buf.end(), p, p + n); };
    auto w32 = [&](int32_t v) { w(&v, 4); };
    const char magic[4] = {'G', 'P', 'U', 'S'};
    w(magic, 4);
    w32(1);
    int nOpes = 0, nMetad = 0, nHills = 0, nPb = 0, nExt = 0;
    for (auto& hb : biases_) {
        nOpes += hb.spec.type == BIAS_OPES;
        nMetad += hb.spec.type == BIAS_METAD;
        nHills += hb.spec.type == BIAS_METAD_HILLS;
        nPb += hb.spec.type == BIAS_PBMETAD;
        nExt += hb.spec.type == BIAS_EXTERNAL;
    }
    w32(nOpes);
    for (auto& hb : biases_) {
        if (hb.spec.type != BIAS_OPES) continue;
        const int D = hb.dev.D;
        int ii[4];
        double dd[1];
        cudaCheck(cudaMemcpy(ii, hb.dev.numKernels, sizeof ii, cudaMemcpyDeviceToHost), "blob");
        cudaCheck(cudaMemcpy(dd, hb.dev.sumUprob, sizeof dd, cudaMemcpyDeviceToHost), "blob");
        int nk = ii[0];
        hb.numKernelsCPU = nk;
        std::vector<double> mean(D), m2(D), c((size_t)nk * D), s((size_t)nk * D), lw(nk);
        cudaCheck(cudaMemcpy(mean.data(), hb.dev.runMean, 8 * D, cudaMemcpyDeviceToHost), "blob");
        cudaCheck(cudaMemcpy(m2.data(), hb.dev.runM2, 8 * D, cudaMemcpyDeviceToHost), "blob");
        if (nk > 0) {
            cudaCheck(cudaMemcpy(c.data(), hb.dev.centers, 8 * c.size(), cudaMemcpyDeviceToHost), "blob");
            cudaCheck(cudaMemcpy(s.data(), hb.dev.sigmas, 8 * s.size(), cudaMemcpyDeviceToHost), "blob");
            cudaCheck(cudaMemcpy(lw.data(), hb.dev.logW, 8 * lw.size(), cudaMemcpyDeviceToHost), "blob");
        }
        w32(nk);
        w(dd, 8);
        w32(ii[3]);  // nSamples
        w(mean.data(), 8 * D);
        w(m2.data(), 8 * D);
        w(c.data(), 8 * c.size());
        w(s.data(), 8 * s.size());
        w(lw.data(), 8 * lw.size());
    }
    w32(0);  // ABMD
    w32(nMetad);
    for (auto& hb : biases_) {
        if (hb.spec.type != BIAS_METAD) continue;
        std::vector<double> g(hb.dev.total);
        cudaCheck(cudaMemcpy(g.data(), hb.dev.grid, 8 * g.size(), cudaMemcpyDeviceToHost), "blob");
        w32(hb.numDeposited);
        w(g.data(), 8 * g.size());
    }
    w32(nPb);
    for (auto& hb : biases_) {
        if (hb.spec.type != BIAS_PBMETAD) continue;
        std::vector<double> g(hb.dev.total);
        cudaCheck(cudaMemcpy(g.data(), hb.dev.grid, 8 * g.size(), cudaMemcpyDeviceToHost), "blob");
        w32(hb.dev.D);
        for (int k = 0; k < hb.dev.D; k++) {
            w32(hb.subDeposited[k]);
            w(g.data() + hb.dev.goff[k], 8 * (size_t)hb.dev.npts[k]);
        }
    }
    w32(nExt);
    for (int k = 0; k < 7; k++) w32(0);  // LINEAR, WALL, OPES_EXPANDED, EXTLAG, EDS, MAXENT, MULTITHERMAL
    if (nHills > 0) {
        const char tag[4] = {'H', 'I', 'L', 'L'};
        w(tag, 4);
        w32(nHills);
        for (auto& hb : biases_) {
            if (hb.spec.type != BIAS_METAD_HILLS) continue;
            int n = 0;
            cudaCheck(cudaMemcpy(&n, hb.dev.hCount, sizeof(int), cudaMemcpyDeviceToHost), "blob");
            std::vector<double> c((size_t)n * hb.dev.D), h(n);
            if (n > 0) {
                cudaCheck(cudaMemcpy(c.data(), hb.dev.hCenters, 8 * c.size(), cudaMemcpyDeviceToHost), "blob");
                cudaCheck(cudaMemcpy(h.data(), hb.dev.hHeights, 8 * h.size(), cudaMemcpyDeviceToHost), "blob");
            }
            w32(n);
            w(c.data(), 8 * c.size());
            w(h.data(), 8 * h.size());
        }
    }
    return buf;
}

void Context::setBiasState(const std::vector<char>& bytes) {
    // CommonSerialization.cpp:180-411: bounds-checked reader, optional header,
    // count checks per section. Deviation: numAllocated is set to the restored
    // kernel count (the reference leaves it at its previous value, so the next
    // append after a restore into a fresh context would claim slot 0).
    if (bytes.empty()) return;
    if (bound_) cudaCheck(cudaStreamSynchronize(stream_), "sync");
    const char* p = bytes.data();
    const char* const end = p + bytes.size();
    auto rd = [&](void* dst, size_t n) {
        if ((size_t)(end - p) < n) throw Error(GLUED_E_CORRUPT, "GLUED bias-state: truncated/corrupt blob");
        std::memcpy(dst, p, n);
        p += n;
    };
    auto more = [&]() { return p < end; };
    if ((size_t)(end - p) >= 8 && std::memcmp(p, "GPUS", 4) == 0) {
        p += 4;
        int32_t ver;
        rd(&ver, 4);
        if (ver != 1) throw Error(GLUED_E_CORRUPT, "GLUED bias-state: unknown blob version");
    }
    int nOpes = 0, nMetad = 0;
    for (auto& hb : biases_) { nOpes += hb.spec.type == BIAS_OPES; nMetad += hb.spec.type == BIAS_METAD; }
    int32_t nb;
    rd(&nb, 4);
    if (nb != nOpes)
        throw Error(GLUED_E_CORRUPT, "GLUED bias-state: OPES bias count mismatch (expected " + std::to_string(nOpes) +
                                         ", got " + std::to_string((long long)nb) + ")");
    for (auto& hb : biases_) {
        if (hb.spec.type != BIAS_OPES) continue;
        const size_t D = hb.dev.D;
        int32_t nk, ns;
        double logZ;
        rd(&nk, 4); rd(&logZ, 8); rd(&ns, 4);
        if (nk < 0 || nk > hb.dev.maxKernels) throw Error(GLUED_E_CORRUPT, "GLUED bias-state: OPES kernel count out of range");
        size_t need = D * 16 + (size_t)nk * D * 16 + (size_t)nk * 8;
        if ((size_t)(end - p) < need) throw Error(GLUED_E_CORRUPT, "GLUED bias-state: truncated/corrupt blob");
        std::vector<double> mean(D), m2(D), c((size_t)nk * D), s((size_t)nk * D), lw(nk);
        rd(mean.data(), 8 * D); rd(m2.data(), 8 * D);
        rd(c.data(), 8 * c.size()); rd(s.data(), 8 * s.size()); rd(lw.data(), 8 * lw.size());
        if (nk > 0) {
            cudaCheck(cudaMemcpy(hb.dev.centers, c.data(), 8 * c.size(), cudaMemcpyHostToDevice), "restore");
            cudaCheck(cudaMemcpy(hb.dev.sigmas, s.data(), 8 * s.size(), cudaMemcpyHostToDevice), "restore");
            cudaCheck(cudaMemcpy(hb.dev.logW, lw.data(), 8 * lw.size(), cudaMemcpyHostToDevice), "restore");
        }
        cudaCheck(cudaMemcpy(hb.dev.runMean, mean.data(), 8 * D, cudaMemcpyHostToDevice), "restore");
        cudaCheck(cudaMemcpy(hb.dev.runM2, m2.data(), 8 * D, cudaMemcpyHostToDevice), "restore");
        int counts[2] = {nk, nk};
        cudaCheck(cudaMemcpy(hb.dev.numKernels, counts, sizeof counts, cudaMemcpyHostToDevice), "restore");
        cudaCheck(cudaMemcpy(hb.dev.nSamples, &ns, 4, cudaMemcpyHostToDevice), "restore");
        cudaCheck(cudaMemcpy(hb.dev.sumUprob, &logZ, 8, cudaMemcpyHostToDevice), "restore");
        // KDNorm = exp(-gamma) + sum exp(logW) (CommonSerialization.cpp:259-265)
        double sumW = std::exp(-hb.dev.gamma);
        for (int k = 0; k < nk; k++) sumW += std::exp(lw[k]);
        cudaCheck(cudaMemcpy(hb.dev.sumWeights, &sumW, 8, cudaMemcpyHostToDevice), "restore");
        hb.numKernelsCPU = nk;
        hb.nSamplesCPU = ns;
    }
    if (more()) {
        int32_t na;
        rd(&na, 4);
        if (na != 0) throw Error(GLUED_E_CORRUPT, "GLUED bias-state: ABMD bias count mismatch (expected 0, got " + std::to_string((long long)na) + ")");
    }
    if (more()) {
        int32_t nm;
        rd(&nm, 4);
        if (nm != nMetad)
            throw Error(GLUED_E_CORRUPT, "GLUED bias-state: MetaD bias count mismatch (expected " + std::to_string(nMetad) +
                                             ", got " + std::to_string((long long)nm) + ")");
        for (auto& hb : biases_) {
            if (hb.spec.type != BIAS_METAD) continue;
            int32_t nd;
            rd(&nd, 4);
            std::vector<double> g(hb.dev.total);
            rd(g.data(), 8 * g.size());
            hb.numDeposited = nd;
            cudaCheck(cudaMemcpy(hb.dev.grid, g.data(), 8 * g.size(), cudaMemcpyHostToDevice), "restore");
        }
    }
    auto atHill = [&]() { return (size_t)(end - p) >= 4 && std::memcmp(p, "HILL", 4) == 0; };
    if (more() && !atHill()) {
        int nPb = 0;
        for (auto& hb : biases_) nPb += hb.spec.type == BIAS_PBMETAD;
        int32_t npb;
        rd(&npb, 4);
        if (npb != nPb)
            throw Error(GLUED_E_CORRUPT, "GLUED bias-state: PBMetaD bias count mismatch (expected " + std::to_string(nPb) +
                                             ", got " + std::to_string((long long)npb) + ")");
        for (auto& hb : biases_) {
            if (hb.spec.type != BIAS_PBMETAD) continue;
            int32_t nsub;
            rd(&nsub, 4);
            if (nsub != hb.dev.D)
                throw Error(GLUED_E_CORRUPT, "GLUED bias-state: PBMetaD sub-grid count mismatch (expected " +
                                                 std::to_string(hb.dev.D) + ", got " + std::to_string((long long)nsub) + ")");
            std::vector<double> g(hb.dev.total);
            std::vector<int> nd(hb.dev.D);
            for (int k = 0; k < hb.dev.D; k++) {
                int32_t n;
                rd(&n, 4);
                nd[k] = n;
                rd(g.data() + hb.dev.goff[k], 8 * (size_t)hb.dev.npts[k]);
            }
            hb.subDeposited = nd;
            cudaCheck(cudaMemcpy(hb.dev.grid, g.data(), 8 * g.size(), cudaMemcpyHostToDevice), "restore");
        }
    }
    // Remaining reference sections: EXTERNAL, LINEAR and WALL are stateless (counts
    // only); the others must be zero for this library's biases.
    const char* names[8] = {"external", "linear", "wall", "OPES_EXPANDED", "extended-Lagrangian", "EDS", "MaxEnt", "OPES multithermal"};
    for (int k = 0; k < 8 && more(); k++) {
        if (atHill()) break;
        int32_t n;
        rd(&n, 4);
        if (n != 0 && k > 2)
            throw Error(GLUED_E_CORRUPT, std::string("GLUED bias-state: ") + names[k] + " bias count mismatch (expected 0, got " + std::to_string((long long)n) + ")");
    }
    if ((size_t)(end - p) >= 8 && std::memcmp(p, "HILL", 4) == 0) {
        p += 4;
        int32_t nh;
        rd(&nh, 4);
        int expect = 0;
        for (auto& hb : biases_) expect += hb.spec.type == BIAS_METAD_HILLS;
        if (nh != expect) throw Error(GLUED_E_CORRUPT, "GLUED bias-state: hill-sum bias count mismatch");
        for (auto& hb : biases_) {
            if (hb.spec.type != BIAS_METAD_HILLS) continue;
            int32_t n;
            rd(&n, 4);
            if (n < 0 || n > hb.dev.maxHills) throw Error(GLUED_E_CORRUPT, "GLUED bias-state: hill count out of range");
            std::vector<double> c((size_t)n * hb.dev.D), h(n);
            rd(c.data(), 8 * c.size()); rd(h.data(), 8 * h.size());
            if (n > 0) {
                cudaCheck(cudaMemcpy(hb.dev.hCenters, c.data(), 8 * c.size(), cudaMemcpyHostToDevice), "restore");
                cudaCheck(cudaMemcpy(hb.dev.hHeights, h.data(), 8 * h.size(), cudaMemcpyHostToDevice), "restore");
            }
            cudaCheck(cudaMemcpy(hb.dev.hCount, &n, 4, cudaMemcpyHostToDevice), "restore");
        }
    }
}

}  // namespace glued
