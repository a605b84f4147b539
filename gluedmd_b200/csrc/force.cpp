// GluedForce descriptor and its XML form.
//
// XML layout follows what OpenMM's XmlSerializer writes for GluedForceProxy
// (serialization/src/GluedForceProxy.cpp:15-79): a root element <Force> whose
// attributes are the node's properties in sorted order (type="GluedForce",
// version, forceGroup, temperature, usesPBC), children <CollectiveVariables>
// with <CV type numAtoms atomN numParams paramN [expression|modelPath]/> and
// <Biases> with <Bias type numCVs cvN numParams paramN numIntParams intParamN/>.
// Doubles are written with 17 significant digits so a round trip is exact.
#include "force.hpp"
#include "../../include/glued_b200.h"

#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <memory>
#include <sstream>

namespace glued {

int GluedForce::addCollectiveVariable(int type, const std::vector<int>& atoms,
                                      const std::vector<double>& params) {
    // GluedForce.cpp:44-61: only the type sign is checked here; everything that
    // needs the System is validated when a context is created.
    if (type < 0)
        throw Error(GLUED_E_INVALID, "GluedForce::addCollectiveVariable: invalid CV type " +
                                         std::to_string(type) + " (must be >= 0)");
    int first = numCVValues_;
    numCVValues_ += (type == CV_PATH) ? 2 : 1;
    CVSpec s;
    s.type = type; s.atoms = atoms; s.params = params;
    cvs_.push_back(s);
    return first;
}

int GluedForce::addExpressionCV(const std::string& expr, const std::vector<int>& inputs) {
    int first = numCVValues_;
    numCVValues_ += 1;
    CVSpec s;
    s.type = CV_EXPRESSION; s.atoms = inputs; s.str = expr;
    cvs_.push_back(s);
    return first;
}

int GluedForce::addPyTorchCV(const std::string& path, const std::vector<int>& atoms,
                             const std::vector<double>& params) {
    int first = numCVValues_;
    numCVValues_ += 1;
    CVSpec s;
    s.type = CV_PYTORCH; s.atoms = atoms; s.params = params; s.str = path;
    cvs_.push_back(s);
    return first;
}

int GluedForce::addBias(int type, const std::vector<int>& cvs, const std::vector<double>& params,
                        const std::vector<int>& iparams) {
    // GluedForce.cpp:81-105: CV indices refer to value slots, not specs.
    int bi = (int)biases_.size();
    for (int c : cvs)
        if (c < 0 || c >= numCVValues_)
            throw Error(GLUED_E_INVALID, "GluedForce::addBias: bias " + std::to_string(bi) + " (type " +
                                             std::to_string(type) + ") references CV value index " +
                                             std::to_string(c) + ", which is out of range [0, " +
                                             std::to_string(numCVValues_) + ")");
    BiasSpec b;
    b.type = type; b.cvs = cvs; b.params = params; b.iparams = iparams;
    biases_.push_back(b);
    return bi;
}

const CVSpec& GluedForce::cv(int i) const {
    if (i < 0 || i >= (int)cvs_.size()) throw Error(GLUED_E_INVALID, "GluedForce: CV index out of range");
    return cvs_[i];
}

const BiasSpec& GluedForce::bias(int i) const {
    if (i < 0 || i >= (int)biases_.size()) throw Error(GLUED_E_INVALID, "GluedForce: bias index out of range");
    return biases_[i];
}

// ------------------------------------------------------------------ XML writer
namespace {

std::string fmtDouble(double v) {
    char buf[40];
    std::snprintf(buf, sizeof buf, "%.17g", v);
    return buf;
}

std::string esc(const std::string& s) {
    std::string o;
    for (char c : s) {
        switch (c) {
            case '&': o += "&amp;"; break;
            case '<': o += "&lt;"; break;
            case '>': o += "&gt;"; break;
            case '"': o += "&quot;"; break;
            default: o += c;
        }
    }
    return o;
}

struct Node {
    std::string name;
    std::map<std::string, std::string> props;
    std::vector<std::unique_ptr<Node>> children;
    Node& child(const std::string& n) {
        children.emplace_back(new Node());
        children.back()->name = n;
        return *children.back();
    }
};

void writeNode(const Node& n, std::ostringstream& out, int depth) {
    out << std::string(depth, '\t') << '<' << n.name;
    for (auto& kv : n.props) out << ' ' << kv.first << "=\"" << esc(kv.second) << '"';
    if (n.children.empty()) { out << "/>\n"; return; }
    out << ">\n";
    for (auto& c : n.children) writeNode(*c, out, depth + 1);
    out << std::string(depth, '\t') << "</" << n.name << ">\n";
}

// Minimal parser for the element/attribute subset above.
struct Parser {
    const std::string& s;
    size_t i = 0;
    explicit Parser(const std::string& str) : s(str) {}
    [[noreturn]] void fail(const std::string& m) {
        throw Error(GLUED_E_INVALID, "GluedForce XML: " + m + " at offset " + std::to_string(i));
    }
    void ws() { while (i < s.size() && std::isspace((unsigned char)s[i])) i++; }
    void skipMisc() {
        for (;;) {
            ws();
            if (s.compare(i, 2, "<?") == 0) { size_t e = s.find("?>", i); if (e == std::string::npos) fail("bad prolog"); i = e + 2; }
            else if (s.compare(i, 4, "<!--") == 0) { size_t e = s.find("-->", i); if (e == std::string::npos) fail("bad comment"); i = e + 3; }
            else return;
        }
    }
    std::string name() {
        size_t b = i;
        while (i < s.size() && (std::isalnum((unsigned char)s[i]) || s[i] == '_' || s[i] == '-' || s[i] == ':' || s[i] == '.')) i++;
        if (b == i) fail("expected a name");
        return s.substr(b, i - b);
    }
    static std::string unesc(const std::string& v) {
        std::string o;
        for (size_t k = 0; k < v.size(); k++) {
            if (v[k] != '&') { o += v[k]; continue; }
            size_t e = v.find(';', k);
            std::string ent = v.substr(k + 1, e - k - 1);
            if (ent == "amp") o += '&'; else if (ent == "lt") o += '<'; else if (ent == "gt") o += '>';
            else if (ent == "quot") o += '"'; else if (ent == "apos") o += '\'';
            else if (!ent.empty() && ent[0] == '#') o += (char)std::strtol(ent.c_str() + 1 + (ent[1] == 'x'), nullptr, ent[1] == 'x' ? 16 : 10);
            k = e;
        }
        return o;
    }
    std::unique_ptr<Node> element() {
        skipMisc();
        if (i >= s.size() || s[i] != '<') fail("expected '<'");
        i++;
        std::unique_ptr<Node> n(new Node());
        n->name = name();
        for (;;) {
            ws();
            if (i >= s.size()) fail("unterminated element");
            if (s[i] == '/') { if (s.compare(i, 2, "/>") != 0) fail("bad '/'"); i += 2; return n; }
            if (s[i] == '>') { i++; break; }
            std::string k = name();
            ws();
            if (i >= s.size() || s[i] != '=') fail("expected '='");
            i++; ws();
            char q = s[i];
            if (q != '"' && q != '\'') fail("expected quote");
            size_t e = s.find(q, i + 1);
            if (e == std::string::npos) fail("unterminated attribute");
            n->props[k] = unesc(s.substr(i + 1, e - i - 1));
            i = e + 1;
        }
        for (;;) {
            skipMisc();
            if (s.compare(i, 2, "</") == 0) {
                i += 2;
                std::string cn = name();
                if (cn != n->name) fail("mismatched closing tag " + cn);
                ws();
                if (i >= s.size() || s[i] != '>') fail("expected '>'");
                i++;
                return n;
            }
            if (i < s.size() && s[i] == '<') { n->children.push_back(element()); continue; }
            size_t e = s.find('<', i);  // text content is ignored
            if (e == std::string::npos) fail("unterminated element " + n->name);
            i = e;
        }
    }
};

const std::string& prop(const Node& n, const std::string& k) {
    auto it = n.props.find(k);
    if (it == n.props.end()) throw Error(GLUED_E_INVALID, "GluedForce XML: missing property '" + k + "' on <" + n.name + ">");
    return it->second;
}
int iprop(const Node& n, const std::string& k) { return std::atoi(prop(n, k).c_str()); }
int iprop(const Node& n, const std::string& k, int def) {
    auto it = n.props.find(k);
    return it == n.props.end() ? def : std::atoi(it->second.c_str());
}
double dprop(const Node& n, const std::string& k) { return std::strtod(prop(n, k).c_str(), nullptr); }
double dprop(const Node& n, const std::string& k, double def) {
    auto it = n.props.find(k);
    return it == n.props.end() ? def : std::strtod(it->second.c_str(), nullptr);
}
bool bprop(const Node& n, const std::string& k, bool def) {
    auto it = n.props.find(k);
    if (it == n.props.end()) return def;
    const std::string& v = it->second;
    return v == "1" || v == "true" || v == "True";
}
const Node* childNamed(const Node& n, const std::string& name) {
    for (auto& c : n.children) if (c->name == name) return c.get();
    return nullptr;
}

}  // namespace

std::string GluedForce::toXml() const {
    // GluedForceProxy::serialize (serialization/src/GluedForceProxy.cpp:15-79).
    Node root;
    root.name = "Force";
    root.props["type"] = "GluedForce";
    root.props["version"] = "1";
    root.props["forceGroup"] = std::to_string(forceGroup);
    root.props["temperature"] = fmtDouble(temperature);
    root.props["usesPBC"] = usesPBC ? "1" : "0";
    Node& cvsN = root.child("CollectiveVariables");
    for (auto& c : cvs_) {
        Node& n = cvsN.child("CV");
        n.props["type"] = std::to_string(c.type);
        n.props["numAtoms"] = std::to_string(c.atoms.size());
        for (size_t j = 0; j < c.atoms.size(); j++) n.props["atom" + std::to_string(j)] = std::to_string(c.atoms[j]);
        n.props["numParams"] = std::to_string(c.params.size());
        for (size_t j = 0; j < c.params.size(); j++) n.props["param" + std::to_string(j)] = fmtDouble(c.params[j]);
        if (c.type == CV_EXPRESSION) n.props["expression"] = c.str;
        else if (c.type == CV_PYTORCH) n.props["modelPath"] = c.str;
    }
    Node& bN = root.child("Biases");
    for (auto& b : biases_) {
        Node& n = bN.child("Bias");
        n.props["type"] = std::to_string(b.type);
        n.props["numCVs"] = std::to_string(b.cvs.size());
        for (size_t j = 0; j < b.cvs.size(); j++) n.props["cv" + std::to_string(j)] = std::to_string(b.cvs[j]);
        n.props["numParams"] = std::to_string(b.params.size());
        for (size_t j = 0; j < b.params.size(); j++) n.props["param" + std::to_string(j)] = fmtDouble(b.params[j]);
        n.props["numIntParams"] = std::to_string(b.iparams.size());
        for (size_t j = 0; j < b.iparams.size(); j++) n.props["intParam" + std::to_string(j)] = std::to_string(b.iparams[j]);
    }
    std::ostringstream out;
    out << "<?xml version=\"1.0\" ?>\n";
    writeNode(root, out, 0);
    return out.str();
}

GluedForce GluedForce::fromXml(const std::string& xml) {
    // GluedForceProxy::deserialize (serialization/src/GluedForceProxy.cpp:81-138).
    Parser p(xml);
    std::unique_ptr<Node> root = p.element();
    auto ti = root->props.find("type");
    if (ti != root->props.end() && ti->second != "GluedForce")
        throw Error(GLUED_E_INVALID, "GluedForce XML: root type is '" + ti->second + "', expected GluedForce");
    if (iprop(*root, "version") != 1)
        throw Error(GLUED_E_INVALID, "GluedForceProxy: unsupported format version");
    GluedForce f;
    f.forceGroup = iprop(*root, "forceGroup", 0);
    f.temperature = dprop(*root, "temperature", -1.0);
    f.usesPBC = bprop(*root, "usesPBC", false);
    const Node* cvsN = childNamed(*root, "CollectiveVariables");
    if (!cvsN) throw Error(GLUED_E_INVALID, "GluedForce XML: missing <CollectiveVariables>");
    for (auto& c : cvsN->children) {
        int type = iprop(*c, "type");
        int na = iprop(*c, "numAtoms");
        std::vector<int> atoms(na);
        for (int j = 0; j < na; j++) atoms[j] = iprop(*c, "atom" + std::to_string(j));
        int np = iprop(*c, "numParams");
        std::vector<double> params(np);
        for (int j = 0; j < np; j++) params[j] = dprop(*c, "param" + std::to_string(j));
        if (type == CV_EXPRESSION) f.addExpressionCV(prop(*c, "expression"), atoms);
        else if (type == CV_PYTORCH) f.addPyTorchCV(prop(*c, "modelPath"), atoms, params);
        else f.addCollectiveVariable(type, atoms, params);
    }
    const Node* bN = childNamed(*root, "Biases");
    if (!bN) throw Error(GLUED_E_INVALID, "GluedForce XML: missing <Biases>");
    for (auto& b : bN->children) {
        int type = iprop(*b, "type");
        int nc = iprop(*b, "numCVs");
        std::vector<int> cvs(nc);
        for (int j = 0; j < nc; j++) cvs[j] = iprop(*b, "cv" + std::to_string(j));
        int np = iprop(*b, "numParams");
        std::vector<double> params(np);
        for (int j = 0; j < np; j++) params[j] = dprop(*b, "param" + std::to_string(j));
        int ni = iprop(*b, "numIntParams");
        std::vector<int> ip(ni);
        for (int j = 0; j < ni; j++) ip[j] = iprop(*b, "intParam" + std::to_string(j));
        f.addBias(type, cvs, params, ip);
    }
    return f;
}

}  // namespace glued
