// extern "C" boundary of include/glued_b200.h. Every entry point converts C++
// exceptions into a status code and keeps the message for glued_last_error().
#include "../../include/glued_b200.h"

#include <algorithm>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "batch.hpp"
#include "context.hpp"
#include "force.hpp"
#include "kernels.hpp"

struct glued_force { glued::GluedForce f; };
struct glued_context { glued::Context* c; };
struct glued_batch { glued::Batch* b; };

namespace {
thread_local std::string g_err;

template <class F>
int guard(F&& fn) {
    try {
        fn();
        g_err.clear();
        return GLUED_OK;
    } catch (const glued::Error& e) {
        g_err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_err = "out of host memory";
        return GLUED_E_INVALID;
    } catch (const std::exception& e) {
        g_err = e.what();
        return GLUED_E_INVALID;
    } catch (...) {
        g_err = "unknown error";
        return GLUED_E_INVALID;
    }
}

void need(const void* p, const char* what) {
    if (!p) throw glued::Error(GLUED_E_INVALID, std::string("null argument: ") + what);
}

template <class T>
void copyOut(const std::vector<T>& v, T* out, int* n, const char* what) {
    need(n, what);
    if (out) {
        if (*n < (int)v.size())
            throw glued::Error(GLUED_E_INVALID, std::string(what) + ": buffer too small (need " + std::to_string(v.size()) + ")");
        if (!v.empty()) std::memcpy(out, v.data(), sizeof(T) * v.size());
    }
    *n = (int)v.size();
}

void copyStr(const std::string& s, char* buf, size_t* len) {
    need(len, "len");
    size_t need_ = s.size() + 1;
    if (buf) {
        if (*len < need_) throw glued::Error(GLUED_E_INVALID, "string buffer too small (need " + std::to_string(need_) + ")");
        std::memcpy(buf, s.c_str(), need_);
    }
    *len = need_;
}
}  // namespace

extern "C" {

const char* glued_last_error(void) { return g_err.c_str(); }
const char* glued_version(void) { return "glued-b200 0.1 (sm_100a)"; }

int glued_force_create(glued_force** out) {
    return guard([&] { need(out, "out"); *out = new glued_force(); });
}
int glued_force_copy(const glued_force* src, glued_force** out) {
    return guard([&] { need(src, "src"); need(out, "out"); *out = new glued_force(*src); });
}
int glued_force_destroy(glued_force* f) {
    return guard([&] { delete f; });
}
int glued_force_add_cv(glued_force* f, int type, const int* atoms, int n_atoms, const double* params, int n_params,
                       int* out_index) {
    return guard([&] {
        need(f, "force");
        std::vector<int> a(atoms, atoms + (atoms ? n_atoms : 0));
        std::vector<double> p(params, params + (params ? n_params : 0));
        int idx = f->f.addCollectiveVariable(type, a, p);
        if (out_index) *out_index = idx;
    });
}
int glued_force_add_bias(glued_force* f, int type, const int* cv, int n_cvs, const double* params, int n_params,
                         const int* ip, int n_ip, int* out_index) {
    return guard([&] {
        need(f, "force");
        int idx = f->f.addBias(type, std::vector<int>(cv, cv + (cv ? n_cvs : 0)),
                               std::vector<double>(params, params + (params ? n_params : 0)),
                               std::vector<int>(ip, ip + (ip ? n_ip : 0)));
        if (out_index) *out_index = idx;
    });
}
int glued_force_add_expression_cv(glued_force* f, const char* expression, const int* inputs, int n_inputs,
                                  int* out_index) {
    return guard([&] {
        need(f, "force"); need(expression, "expression");
        int idx = f->f.addExpressionCV(expression, std::vector<int>(inputs, inputs + (inputs ? n_inputs : 0)));
        if (out_index) *out_index = idx;
    });
}
int glued_force_add_pytorch_cv(glued_force* f, const char* path, const int* atoms, int n_atoms, const double* params,
                               int n_params, int* out_index) {
    return guard([&] {
        need(f, "force"); need(path, "model_path");
        int idx = f->f.addPyTorchCV(path, std::vector<int>(atoms, atoms + (atoms ? n_atoms : 0)),
                                    std::vector<double>(params, params + (params ? n_params : 0)));
        if (out_index) *out_index = idx;
    });
}
int glued_force_num_cv_values(const glued_force* f, int* out) {
    return guard([&] { need(f, "force"); need(out, "out"); *out = f->f.numCVValues(); });
}
int glued_force_num_cv_specs(const glued_force* f, int* out) {
    return guard([&] { need(f, "force"); need(out, "out"); *out = f->f.numCVSpecs(); });
}
int glued_force_num_biases(const glued_force* f, int* out) {
    return guard([&] { need(f, "force"); need(out, "out"); *out = f->f.numBiases(); });
}
int glued_force_get_cv(const glued_force* f, int idx, int* type, int* atoms, int* n_atoms, double* params,
                       int* n_params) {
    return guard([&] {
        need(f, "force");
        const glued::CVSpec& c = f->f.cv(idx);
        if (type) *type = c.type;
        copyOut(c.atoms, atoms, n_atoms, "atoms");
        copyOut(c.params, params, n_params, "params");
    });
}
int glued_force_get_cv_string(const glued_force* f, int idx, char* buf, size_t* len) {
    return guard([&] { need(f, "force"); copyStr(f->f.cv(idx).str, buf, len); });
}
int glued_force_get_bias(const glued_force* f, int idx, int* type, int* cvs, int* n_cvs, double* params, int* n_params,
                         int* ip, int* n_ip) {
    return guard([&] {
        need(f, "force");
        const glued::BiasSpec& b = f->f.bias(idx);
        if (type) *type = b.type;
        copyOut(b.cvs, cvs, n_cvs, "cv_indices");
        copyOut(b.params, params, n_params, "params");
        copyOut(b.iparams, ip, n_ip, "int_params");
    });
}
int glued_force_set_temperature(glued_force* f, double k) { return guard([&] { need(f, "force"); f->f.temperature = k; }); }
int glued_force_get_temperature(const glued_force* f, double* k) {
    return guard([&] { need(f, "force"); need(k, "out"); *k = f->f.temperature; });
}
int glued_force_set_pbc(glued_force* f, int yes) { return guard([&] { need(f, "force"); f->f.usesPBC = yes != 0; }); }
int glued_force_get_pbc(const glued_force* f, int* yes) {
    return guard([&] { need(f, "force"); need(yes, "out"); *yes = f->f.usesPBC ? 1 : 0; });
}
int glued_force_set_force_group(glued_force* f, int g) {
    return guard([&] {
        need(f, "force");
        if (g < 0 || g > 31) throw glued::Error(GLUED_E_INVALID, "Force group must be between 0 and 31");
        f->f.forceGroup = g;
    });
}
int glued_force_get_force_group(const glued_force* f, int* g) {
    return guard([&] { need(f, "force"); need(g, "out"); *g = f->f.forceGroup; });
}
int glued_force_set_test_force(glued_force* f, int mode, double scale) {
    return guard([&] { need(f, "force"); f->f.testForceMode = mode; f->f.testForceScale = scale; });
}
int glued_force_get_test_force(const glued_force* f, int* mode, double* scale) {
    return guard([&] {
        need(f, "force");
        if (mode) *mode = f->f.testForceMode;
        if (scale) *scale = f->f.testForceScale;
    });
}
int glued_force_set_test_bias_gradients(glued_force* f, const double* g, int n) {
    return guard([&] { need(f, "force"); f->f.testBiasGradients.assign(g, g + (g ? n : 0)); });
}
int glued_force_get_test_bias_gradients(const glued_force* f, double* g, int* n) {
    return guard([&] { need(f, "force"); copyOut(f->f.testBiasGradients, g, n, "gradients"); });
}
int glued_force_serialize_xml(const glued_force* f, char* buf, size_t* len) {
    return guard([&] { need(f, "force"); copyStr(f->f.toXml(), buf, len); });
}
int glued_force_deserialize_xml(const char* xml, glued_force** out) {
    return guard([&] {
        need(xml, "xml"); need(out, "out");
        glued::GluedForce f = glued::GluedForce::fromXml(xml);
        *out = new glued_force{f};
    });
}

// ---------------------------------------------------------------- context
int glued_context_create(const glued_force* f, int num_particles, const double* masses, glued_context** out) {
    return guard([&] {
        need(f, "force"); need(out, "out");
        *out = new glued_context{new glued::Context(f->f, num_particles, masses)};
    });
}
int glued_context_destroy(glued_context* c) {
    return guard([&] {
        if (c) { delete c->c; delete c; }
    });
}
int glued_context_bind(glued_context* c, void* stream, const void* posq, const int* atom_index, long long* force_buffer,
                       int padded) {
    return guard([&] {
        need(c, "context"); need(posq, "posq"); need(force_buffer, "force_buffer");
        c->c->bind((cudaStream_t)stream, posq, atom_index, force_buffer, padded);
    });
}
int glued_context_atoms_reordered(glued_context* c) {
    return guard([&] { need(c, "context"); c->c->atomsReordered(); });
}
int glued_context_set_box(glued_context* c, const double box[9]) {
    return guard([&] { need(c, "context"); need(box, "box"); c->c->setBox(box); });
}
int glued_context_set_step(glued_context* c, long long step) {
    return guard([&] { need(c, "context"); c->c->setStep(step); });
}
int glued_context_execute(glued_context* c, int include_forces, int include_energy, double* energy_out) {
    return guard([&] {
        need(c, "context");
        double e = c->c->execute(include_forces != 0, include_energy != 0);
        if (energy_out) *energy_out = e;
    });
}
int glued_context_update_state(glued_context* c, int step) {
    return guard([&] { need(c, "context"); c->c->updateState(step); });
}
int glued_context_get_cv_values(glued_context* c, double* out, int n) {
    return guard([&] {
        need(c, "context");
        std::vector<double> v = c->c->cvValues();
        if (n < (int)v.size()) throw glued::Error(GLUED_E_INVALID, "cv buffer too small (need " + std::to_string(v.size()) + ")");
        if (!v.empty()) { need(out, "out"); std::memcpy(out, v.data(), sizeof(double) * v.size()); }
    });
}
int glued_context_get_last_bias(glued_context* c, double* out) {
    return guard([&] { need(c, "context"); need(out, "out"); *out = c->c->lastBias(); });
}
int glued_context_get_bias_state(glued_context* c, char* buf, size_t* len) {
    return guard([&] {
        need(c, "context"); need(len, "len");
        std::vector<char> b = c->c->getBiasState();
        if (buf) {
            if (*len < b.size()) throw glued::Error(GLUED_E_INVALID, "bias-state buffer too small (need " + std::to_string(b.size()) + ")");
            std::memcpy(buf, b.data(), b.size());
        }
        *len = b.size();
    });
}
int glued_context_set_bias_state(glued_context* c, const char* buf, size_t len) {
    return guard([&] {
        need(c, "context");
        std::vector<char> b(buf, buf + (buf ? len : 0));
        c->c->setBiasState(b);
    });
}
int glued_context_opes_metrics(glued_context* c, int idx, double out[4]) {
    return guard([&] {
        need(c, "context"); need(out, "out");
        std::vector<double> m = c->c->opesMetrics(idx);
        for (int i = 0; i < 4; i++) out[i] = m[i];
    });
}
int glued_context_kernel_sigmas(glued_context* c, int idx, float* out, int* n) {
    return guard([&] { need(c, "context"); copyOut(c->c->kernelSigmas(idx), out, n, "sigmas"); });
}
int glued_context_multiwalker_ptrs(glued_context* c, int bias_index, long long* out, int* n) {
    return guard([&] { need(c, "context"); copyOut(c->c->multiWalkerPtrs(bias_index), out, n, "ptrs"); });
}
int glued_context_set_multiwalker_ptrs(glued_context* c, int bias_index, const long long* ptrs, int n) {
    return guard([&] {
        need(c, "context");
        c->c->setMultiWalkerPtrs(bias_index, std::vector<long long>(ptrs, ptrs + (ptrs ? n : 0)));
    });
}
int glued_context_device_arrays(glued_context* c, void** cvv, void** dudcv, void** ja, void** jx, void** jy, void** jz,
                                void** jc, int* num_cvs, int* num_rows) {
    return guard([&] {
        need(c, "context");
        const glued::JacDev& J = c->c->jac();
        if (cvv) *cvv = c->c->dCV();
        if (dudcv) *dudcv = c->c->dGrad();
        if (ja) *ja = J.atom;
        if (jx) *jx = J.gx;
        if (jy) *jy = J.gy;
        if (jz) *jz = J.gz;
        if (jc) *jc = J.cv;
        if (num_cvs) *num_cvs = c->c->numCVs();
        if (num_rows) *num_rows = c->c->numRows();
    });
}
int glued_context_profile_phases(glued_context* c, int reps, double* out, int* n) {
    return guard([&] { need(c, "context"); copyOut(c->c->profilePhases(reps), out, n, "phases"); });
}
int glued_context_launch_count(glued_context* c, long long* count) {
    return guard([&] { need(c, "context"); need(count, "out"); *count = c->c->launchCount(); });
}
int glued_measure_hill_staging(int num_hills, int ctas, int reps, double out[2], int* status) {
    return guard([&] {
        need(out, "out"); need(status, "status");
        glued::measureHillStaging(num_hills, ctas, reps, &out[0], &out[1], status);
    });
}
int glued_measure_fp32_peak(double* tflops) {
    return guard([&] { need(tflops, "out"); *tflops = glued::measureFp32Peak(); });
}
int glued_ad_forward(int dtype, void* stream, const glued_ad_spec* spec, double* out, double* partials,
                     int n_partials) {
    return guard([&] {
        need(spec, "spec"); need(out, "out"); need(partials, "partials");
        if (n_partials < 1) throw glued::Error(GLUED_E_INVALID, "n_partials must be >= 1");
        glued::adForward(dtype, (cudaStream_t)stream, *spec, out, partials, n_partials);
    });
}
int glued_ad_backward(int dtype, void* stream, const glued_ad_spec* spec, const double* out,
                      const double* grad_energy, long long* acc, void* grad_pos, void* grad_r0, void* grad_frames,
                      void* grad_heights) {
    return guard([&] {
        need(spec, "spec"); need(out, "out"); need(grad_energy, "grad_energy"); need(acc, "acc");
        need(grad_pos, "grad_pos"); need(grad_r0, "grad_r0"); need(grad_frames, "grad_frames");
        need(grad_heights, "grad_heights");
        glued::adBackward(dtype, (cudaStream_t)stream, *spec, out, grad_energy, acc, grad_pos, grad_r0, grad_frames,
                          grad_heights);
    });
}
int glued_coordination_noalloc(void* stream, const void* posq, const int* group_a, int n_a, const int* group_b,
                               int n_b, double r0, double n, double m, int periodic, const double box[9],
                               double* cn_out, float* grad_out) {
    return guard([&] {
        glued::coordinationNoAlloc((cudaStream_t)stream, posq, group_a, n_a, group_b, n_b, r0, n, m, periodic, box,
                                   cn_out, grad_out);
    });
}
int glued_context_opes_last_decision(glued_context* c, int idx, int* decision) {
    return guard([&] { need(c, "context"); need(decision, "out"); *decision = c->c->opesLastDecision(idx); });
}
int glued_context_coordination_pairs(glued_context* c, int cv_index, int* out, long long cap, long long* n) {
    return guard([&] {
        need(c, "context"); need(n, "out");
        std::vector<int> v = c->c->cellPairs(cv_index);
        *n = (long long)(v.size() / 2);
        if (out && cap > 0) std::memcpy(out, v.data(), sizeof(int) * 2 * (size_t)std::min<long long>(cap, *n));
    });
}
int glued_context_set_sum_precision(glued_context* c, int kernel_sums, int coordination) {
    return guard([&] { need(c, "context"); c->c->setSumPrecision(kernel_sums, coordination); });
}
int glued_context_get_sum_precision(glued_context* c, int* kernel_sums, int* coordination) {
    return guard([&] {
        need(c, "context"); need(kernel_sums, "out"); need(coordination, "out");
        *kernel_sums = c->c->sumMode();
        *coordination = c->c->coordBlocked() ? 1 : 0;
    });
}

// ------------------------------------------------------------------ batch
int glued_batch_create(const glued_force* const* forces, int num_walkers, const glued_walker_desc* walkers,
                       glued_batch** out) {
    return guard([&] {
        need(forces, "forces"); need(walkers, "walkers"); need(out, "out");
        if (num_walkers < 1) throw glued::Error(GLUED_E_INVALID, "num_walkers must be >= 1");
        std::vector<const glued::GluedForce*> fs;
        for (int w = 0; w < num_walkers; w++) { need(forces[w], "forces[w]"); fs.push_back(&forces[w]->f); }
        *out = new glued_batch{new glued::Batch(fs, walkers)};
    });
}
int glued_batch_destroy(glued_batch* b) {
    return guard([&] {
        if (b) { delete b->b; delete b; }
    });
}
int glued_batch_set_stream(glued_batch* b, void* stream) {
    return guard([&] { need(b, "batch"); b->b->setStream((cudaStream_t)stream); });
}
int glued_batch_set_tuning(glued_batch* b, const int tune[4]) {
    return guard([&] {
        need(b, "batch"); need(tune, "tune");
        glued::BatchTuning t;
        t.ra = tune[0]; t.parts = tune[1]; t.plain = tune[2]; t.ch = tune[3] == 0 ? 128 : tune[3];
        b->b->setTuning(t);
    });
}
int glued_batch_get_tuning(glued_batch* b, int tune[4]) {
    return guard([&] {
        need(b, "batch"); need(tune, "tune");
        glued::BatchTuning t = b->b->tuning();
        tune[0] = t.ra; tune[1] = t.parts; tune[2] = t.plain; tune[3] = t.ch;
    });
}
int glued_batch_set_sum_precision(glued_batch* b, int mode) {
    return guard([&] { need(b, "batch"); b->b->setSumPrecision(mode); });
}
int glued_batch_get_sum_precision(glued_batch* b, int* mode) {
    return guard([&] { need(b, "batch"); need(mode, "out"); *mode = b->b->sumPrecision(); });
}
int glued_batch_autotune(glued_batch* b, int tune[4]) { return glued_batch_autotune_ex(b, 1, tune, nullptr); }
int glued_batch_autotune_ex(glued_batch* b, int use_cache, int tune[4], int* cached) {
    return guard([&] {
        need(b, "batch");
        glued::BatchTuning t = b->b->autotune(use_cache != 0);
        if (tune) { tune[0] = t.ra; tune[1] = t.parts; tune[2] = t.plain; tune[3] = t.ch; }
        if (cached) *cached = b->b->lastTuneCached() ? 1 : 0;
    });
}
int glued_batch_execute(glued_batch* b) {
    return guard([&] { need(b, "batch"); b->b->execute(); });
}
int glued_batch_update_state(glued_batch* b, int step) {
    return guard([&] { need(b, "batch"); b->b->updateState(step); });
}
int glued_batch_get_energies(glued_batch* b, double* e) {
    return guard([&] { need(b, "batch"); need(e, "out"); b->b->energies(e); });
}
int glued_batch_get_cv_values(glued_batch* b, double* v) {
    return guard([&] { need(b, "batch"); need(v, "out"); b->b->cvValues(v); });
}
int glued_batch_num_cvs(glued_batch* b, int* n) {
    return guard([&] { need(b, "batch"); need(n, "out"); *n = b->b->numCVs(); });
}
int glued_batch_num_hills(glued_batch* b, int* n) {
    return guard([&] { need(b, "batch"); need(n, "out"); *n = b->b->numHills(); });
}
int glued_batch_set_hills(glued_batch* b, const double* c, const double* h, int n) {
    return guard([&] {
        need(b, "batch");
        if (n > 0) { need(c, "centers"); need(h, "heights"); }
        b->b->setHills(c, h, n);
    });
}
int glued_batch_get_hills(glued_batch* b, double* c, double* h, int n) {
    return guard([&] {
        need(b, "batch");
        if (n > 0) { need(c, "centers"); need(h, "heights"); }
        b->b->getHills(c, h, n);
    });
}
int glued_batch_status(glued_batch* b, int* status) {
    return guard([&] { need(b, "batch"); need(status, "out"); *status = b->b->status(); });
}
int glued_batch_launch_count(glued_batch* b, long long* count) {
    return guard([&] { need(b, "batch"); need(count, "out"); *count = b->b->launchCount(); });
}
int glued_batch_phase_times(glued_batch* b, double* out) {
    return guard([&] { need(b, "batch"); need(out, "out"); b->b->phaseTimes(out); });
}

int glued_batch_phase_stamps(glued_batch* b, unsigned long long* out, long long cap, long long* n) {
    return guard([&] {
        need(b, "batch");
        need(n, "n");
        if (cap < 0) throw glued::Error(GLUED_E_INVALID, "cap must be >= 0");
        *n = b->b->phaseStamps(cap > 0 ? out : nullptr, cap);
    });
}

}  // extern "C"
