// ORACLE — test infrastructure only. Nothing in the product (gluedmd_b200/) may
// link, load or call this file; tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg use it as the checker.
//
// A CPU restatement of GLUED's per-step hot path (CV evaluation -> bias ->
// chain-rule force scatter, plus MetaD/OPES deposition), written from the
// reference's algorithm, not copied from it. Every function is templated on the
// arithmetic type R:
//   R = float  : the reference's FP32 ("real" = float) semantics,
//   R = double : the FP64 oracle used for the relative-error gates.
// Reference citations are relative to the GLUED source tree.
//
// Jacobian rows are produced in the reference's table order
// (platforms/common/src/CommonGluedKernels.cpp:4170-4230): each row is
// (atom, gx, gy, gz, cv). Gradients are returned as double; in FP32 mode they are
// first rounded to float exactly where the reference stores float.
//
// Deterministic FP64 math (exp/log/pow) for the OPES deposit decisions comes from
// gluedmd_b200/csrc/glued_dmath.h, a header compiled identically for host and
// device so that merge decisions can be compared bit for bit.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#include "../gluedmd_b200/csrc/glued_dmath.h"

namespace {

template <class R> struct V3 { R x, y, z; };

// Minimum-image convention, triclinic reduced box, strict z -> y -> x order with
// floor(d/L + 0.5) (CommonGluedKernels.cpp:74-90).
template <class R>
struct Box {
    R inv[3];
    R a[3], b[3], c[3];
    explicit Box(const double* box9) {
        for (int i = 0; i < 3; i++) { a[i] = (R)box9[i]; b[i] = (R)box9[3 + i]; c[i] = (R)box9[6 + i]; }
        inv[0] = (R)(1.0 / box9[0]);
        inv[1] = (R)(1.0 / box9[4]);
        inv[2] = (R)(1.0 / box9[8]);
    }
    V3<R> image(V3<R> d) const {
        R s3 = std::floor(d.z * inv[2] + (R)0.5);
        d.x -= s3 * c[0]; d.y -= s3 * c[1]; d.z -= s3 * c[2];
        R s2 = std::floor(d.y * inv[1] + (R)0.5);
        d.x -= s2 * b[0]; d.y -= s2 * b[1];
        R s1 = std::floor(d.x * inv[0] + (R)0.5);
        d.x -= s1 * a[0];
        return d;
    }
};

template <class R>
inline V3<R> P(const double* pos, int i) {
    // Positions enter as OpenMM posq would hold them: rounded to R.
    return V3<R>{(R)pos[3 * i], (R)pos[3 * i + 1], (R)pos[3 * i + 2]};
}
template <class R> inline V3<R> sub(V3<R> a, V3<R> b) { return V3<R>{a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
    return V3<R>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Storage rounding of a Jacobian component: float in the reference.
template <class R> inline double jstore(R v) { return (double)(float)v; }
template <> inline double jstore<double>(double v) { return v; }

struct Jac {
    int* atom; double* gx; double* gy; double* gz; int* cv;
    void set(int row, int a, double x, double y, double z, int c) {
        atom[row] = a; gx[row] = x; gy[row] = y; gz[row] = z; cv[row] = c;
    }
};

// ---------------------------------------------------------------- CVs

// Distance: CommonGluedKernels.cpp:177-229.
template <class R>
void cv_distance(const double* pos, const int* pairs, int n, int cv0, int jac0,
                 const double* box9, int periodic, double* cvv, Jac J) {
    Box<R> box(box9);
    for (int i = 0; i < n; i++) {
        int a = pairs[2 * i], b = pairs[2 * i + 1];
        V3<R> d = sub(P<R>(pos, b), P<R>(pos, a));
        if (periodic) d = box.image(d);
        R r = std::sqrt(dot(d, d));
        R inv = r > (R)1e-10 ? (R)1 / r : (R)0;
        cvv[cv0 + i] = (double)r;
        J.set(jac0 + 2 * i, a, jstore<R>(-d.x * inv), jstore<R>(-d.y * inv), jstore<R>(-d.z * inv), cv0 + i);
        J.set(jac0 + 2 * i + 1, b, jstore<R>(d.x * inv), jstore<R>(d.y * inv), jstore<R>(d.z * inv), cv0 + i);
    }
}

// Angle at the middle atom: CommonGluedKernels.cpp:238-325.
template <class R>
void cv_angle(const double* pos, const int* trip, int n, int cv0, int jac0,
              const double* box9, int periodic, double* cvv, Jac J) {
    Box<R> box(box9);
    for (int i = 0; i < n; i++) {
        int a = trip[3 * i], b = trip[3 * i + 1], c = trip[3 * i + 2];
        V3<R> pb = P<R>(pos, b);
        V3<R> d1 = sub(P<R>(pos, a), pb), d2 = sub(P<R>(pos, c), pb);
        if (periodic) { d1 = box.image(d1); d2 = box.image(d2); }
        R r1 = std::sqrt(dot(d1, d1)), r2 = std::sqrt(dot(d2, d2));
        R i1 = r1 > (R)1e-10 ? (R)1 / r1 : (R)0;
        R i2 = r2 > (R)1e-10 ? (R)1 / r2 : (R)0;
        V3<R> n1{d1.x * i1, d1.y * i1, d1.z * i1}, n2{d2.x * i2, d2.y * i2, d2.z * i2};
        R ct = dot(n1, n2);
        ct = std::max((R)-1, std::min((R)1, ct));
        R th = std::acos(ct);
        R st = std::sqrt((R)1 - ct * ct);
        R is = st > (R)1e-6 ? (R)1 / st : (R)0;
        cvv[cv0 + i] = (double)th;
        R s1 = i1 * is, s2 = i2 * is;
        V3<R> jA{-(n2.x - ct * n1.x) * s1, -(n2.y - ct * n1.y) * s1, -(n2.z - ct * n1.z) * s1};
        V3<R> jC{-(n1.x - ct * n2.x) * s2, -(n1.y - ct * n2.y) * s2, -(n1.z - ct * n2.z) * s2};
        V3<R> jB{-(jA.x + jC.x), -(jA.y + jC.y), -(jA.z + jC.z)};
        int r0 = jac0 + 3 * i;
        J.set(r0, a, jstore<R>(jA.x), jstore<R>(jA.y), jstore<R>(jA.z), cv0 + i);
        J.set(r0 + 1, b, jstore<R>(jB.x), jstore<R>(jB.y), jstore<R>(jB.z), cv0 + i);
        J.set(r0 + 2, c, jstore<R>(jC.x), jstore<R>(jC.y), jstore<R>(jC.z), cv0 + i);
    }
}

// Dihedral, Blondel-Karplus form: CommonGluedKernels.cpp:335-444.
template <class R>
void cv_dihedral(const double* pos, const int* quad, int n, int cv0, int jac0,
                 const double* box9, int periodic, double* cvv, Jac J) {
    Box<R> box(box9);
    for (int i = 0; i < n; i++) {
        int ia = quad[4 * i], ib = quad[4 * i + 1], ic = quad[4 * i + 2], id = quad[4 * i + 3];
        V3<R> pa = P<R>(pos, ia), pb = P<R>(pos, ib), pc = P<R>(pos, ic), pd = P<R>(pos, id);
        V3<R> b1 = sub(pb, pa), b2 = sub(pc, pb), b3 = sub(pd, pc);
        if (periodic) { b1 = box.image(b1); b2 = box.image(b2); b3 = box.image(b3); }
        V3<R> t = cross(b1, b2), u = cross(b2, b3);
        R d = std::sqrt(dot(b2, b2));
        R t2 = dot(t, t), u2 = dot(u, u);
        R phi = std::atan2(d * dot(b1, u), dot(t, u));
        cvv[cv0 + i] = (double)phi;
        R it2 = t2 > (R)1e-10 ? (R)1 / t2 : (R)0;
        R iu2 = u2 > (R)1e-10 ? (R)1 / u2 : (R)0;
        R id_ = d > (R)1e-10 ? (R)1 / d : (R)0;
        R c1 = dot(b1, b2) * id_;
        R c2 = dot(b3, b2) * id_;
        R aT = d * it2, aU = d * iu2, bTB = (d + c1) * it2, bUB = c2 * iu2;
        V3<R> jA{-aT * t.x, -aT * t.y, -aT * t.z};
        V3<R> jD{aU * u.x, aU * u.y, aU * u.z};
        V3<R> jB{bTB * t.x + bUB * u.x, bTB * t.y + bUB * u.y, bTB * t.z + bUB * u.z};
        V3<R> jC{-(jA.x + jB.x + jD.x), -(jA.y + jB.y + jD.y), -(jA.z + jB.z + jD.z)};
        int r0 = jac0 + 4 * i;
        J.set(r0, ia, jstore<R>(jA.x), jstore<R>(jA.y), jstore<R>(jA.z), cv0 + i);
        J.set(r0 + 1, ib, jstore<R>(jB.x), jstore<R>(jB.y), jstore<R>(jB.z), cv0 + i);
        J.set(r0 + 2, ic, jstore<R>(jC.x), jstore<R>(jC.y), jstore<R>(jC.z), cv0 + i);
        J.set(r0 + 3, id, jstore<R>(jD.x), jstore<R>(jD.y), jstore<R>(jD.z), cv0 + i);
    }
}

// COM distance: CommonGluedKernels.cpp:456-539. `off` is the interleaved
// [g1Start, g2Start, g2End, ...] table (2n+1 entries); masses are float.
template <class R>
void cv_com_distance(const double* pos, const int* off, const int* atoms, const float* mass,
                     const float* totm, int n, int cv0, int jac0, const double* box9,
                     int periodic, double* cvv, Jac J) {
    Box<R> box(box9);
    for (int i = 0; i < n; i++) {
        int s1 = off[2 * i], s2 = off[2 * i + 1], e2 = off[2 * i + 2];
        float m1 = totm[2 * i], m2 = totm[2 * i + 1];
        V3<R> c1{0, 0, 0}, c2{0, 0, 0};
        for (int j = s1; j < s2; j++) {
            V3<R> p = P<R>(pos, atoms[j]); R w = (R)mass[j];
            c1.x += w * p.x; c1.y += w * p.y; c1.z += w * p.z;
        }
        R i1 = (R)1 / (R)m1; c1.x *= i1; c1.y *= i1; c1.z *= i1;
        for (int j = s2; j < e2; j++) {
            V3<R> p = P<R>(pos, atoms[j]); R w = (R)mass[j];
            c2.x += w * p.x; c2.y += w * p.y; c2.z += w * p.z;
        }
        R i2 = (R)1 / (R)m2; c2.x *= i2; c2.y *= i2; c2.z *= i2;
        V3<R> d = sub(c2, c1);
        if (periodic) d = box.image(d);
        R r = std::sqrt(dot(d, d));
        R inv = r > (R)1e-10 ? (R)1 / r : (R)0;
        cvv[cv0 + i] = (double)r;
        for (int j = s1; j < s2; j++) {
            R w = std::is_same<R, float>::value ? (R)(mass[j] / m1) : (R)mass[j] / (R)m1;
            J.set(jac0 + j, atoms[j], jstore<R>(-d.x * inv * w), jstore<R>(-d.y * inv * w),
                  jstore<R>(-d.z * inv * w), cv0 + i);
        }
        for (int j = s2; j < e2; j++) {
            R w = std::is_same<R, float>::value ? (R)(mass[j] / m2) : (R)mass[j] / (R)m2;
            J.set(jac0 + j, atoms[j], jstore<R>(d.x * inv * w), jstore<R>(d.y * inv * w),
                  jstore<R>(d.z * inv * w), cv0 + i);
        }
    }
}

// Radius of gyration, COM without PBC, displacement with PBC:
// CommonGluedKernels.cpp:556-639.
template <class R>
void cv_gyration(const double* pos, const int* off, const int* atoms, const float* mass,
                 const float* totm, int n, int cv0, int jac0, const double* box9, int periodic,
                 double* cvv, Jac J) {
    Box<R> box(box9);
    for (int i = 0; i < n; i++) {
        int s = off[i], e = off[i + 1];
        float M = totm[i];
        R invM = (R)1 / (R)M;
        V3<R> com{0, 0, 0};
        for (int j = s; j < e; j++) {
            V3<R> p = P<R>(pos, atoms[j]); R m = (R)mass[j];
            com.x += m * p.x; com.y += m * p.y; com.z += m * p.z;
        }
        com.x *= invM; com.y *= invM; com.z *= invM;
        R rg2 = 0;
        std::vector<V3<R>> dr(e - s);
        for (int j = s; j < e; j++) {
            V3<R> d = sub(P<R>(pos, atoms[j]), com);
            if (periodic) d = box.image(d);
            rg2 += (R)mass[j] * dot(d, d);
            dr[j - s] = d;
        }
        rg2 *= invM;
        R rg = std::sqrt(rg2);
        R irg = rg > (R)1e-10 ? (R)1 / rg : (R)0;
        cvv[cv0 + i] = (double)rg;
        for (int j = s; j < e; j++) {
            V3<R> d = dr[j - s];
            if (std::is_same<R, float>::value) {
                // The reference caches the displacement as float for <= 256 atoms
                // (CommonGluedKernels.cpp:595-617); for float R that is exact.
            }
            R w = std::is_same<R, float>::value ? (R)(mass[j] / M) : (R)mass[j] / (R)M;
            J.set(jac0 + j, atoms[j], jstore<R>(w * d.x * irg), jstore<R>(w * d.y * irg),
                  jstore<R>(w * d.z * irg), cv0 + i);
        }
    }
}

// Rational switch (1-x^n)/(1-x^m) with the reference's Taylor branch near x=1,
// returns f and df/dr: CommonGluedKernels.cpp:969-1010.
template <class R>
inline bool coord_switch(R r, R r0, R rn, R rm, R preRes, R preDf, R preSec, R& f, R& dfdr) {
    R x = r / r0;
    if (x > (R)1000) return false;
    R dx1 = x - (R)1;
    if (std::fabs(dx1) < (R)1e-4) {
        f = preRes + dx1 * (preDf + (R)0.5 * dx1 * preSec);
        dfdr = (preDf + dx1 * preSec) / r0;
    } else if (x < (R)1e-10) {
        f = 1; dfdr = 0;
    } else {
        R xn = std::pow(x, rn), xm = std::pow(x, rm);
        R den = (R)1 - xm;
        f = ((R)1 - xn) / den;
        R dfx = (rm * (xm / x) - rn * (xn / x) + (rn - rm) * (xn * xm / x)) / (den * den);
        dfdr = dfx / r0;
    }
    return true;
}

// Coordination number, all ng1 x ng2 minimum-image pairs, no cutoff:
// CommonGluedKernels.cpp:899-1031. off = [g1Start, g2Start, g2End] per CV;
// params = [r0, n, m] (float). Optional cutoff (rc > 0) is this build's
// extension and has no reference counterpart.
template <class R>
void cv_coordination(const double* pos, const int* off, const int* atoms, const float* prm,
                     int n, int cv0, int jac0, const double* box9, int periodic, double rc,
                     double* cvv, Jac J) {
    Box<R> box(box9);
    for (int i = 0; i < n; i++) {
        int s1 = off[2 * i], s2 = off[2 * i + 1], e2 = off[2 * i + 2];
        R r0 = (R)prm[3 * i], rn = (R)prm[3 * i + 1], rm = (R)prm[3 * i + 2];
        R preRes = rn / rm;
        R preDf = (R)0.5 * rn * (rn - rm) / rm;
        R preSec = rn * (rm * rm - (R)3 * rm * (rn - (R)1) + rn * ((R)2 * rn - (R)3)) / ((R)6 * rm);
        std::vector<R> gx(e2 - s1, 0), gy(e2 - s1, 0), gz(e2 - s1, 0);
        std::vector<V3<R>> pl(e2 - s2);
        for (int l = s2; l < e2; l++) pl[l - s2] = P<R>(pos, atoms[l]);
        R cn = 0;
        R rc2 = (R)(rc * rc);
        for (int k = s1; k < s2; k++) {
            V3<R> pk = P<R>(pos, atoms[k]);
            for (int l = s2; l < e2; l++) {
                V3<R> d = sub(pk, pl[l - s2]);
                if (periodic) d = box.image(d);
                R r2 = dot(d, d);
                if (r2 < (R)1e-20) continue;
                if (rc > 0 && r2 >= rc2) continue;
                R r = std::sqrt(r2);
                R f, dfdr;
                if (!coord_switch<R>(r, r0, rn, rm, preRes, preDf, preSec, f, dfdr)) continue;
                cn += f;
                R ir = (R)1 / r;
                R cx = dfdr * d.x * ir, cy = dfdr * d.y * ir, cz = dfdr * d.z * ir;
                if (std::is_same<R, float>::value) { cx = (float)cx; cy = (float)cy; cz = (float)cz; }
                gx[k - s1] += cx; gy[k - s1] += cy; gz[k - s1] += cz;
                gx[l - s1] -= cx; gy[l - s1] -= cy; gz[l - s1] -= cz;
            }
        }
        cvv[cv0 + i] = (double)cn;
        for (int j = s1; j < e2; j++)
            J.set(jac0 + j, atoms[j], jstore<R>(gx[j - s1]), jstore<R>(gy[j - s1]), jstore<R>(gz[j - s1]), cv0 + i);
    }
}

// No-fit RMSD: CommonGluedKernels.cpp:810-881. ref is float[3*total].
template <class R>
void cv_rmsd(const double* pos, const int* off, const int* atoms, const float* ref, int n,
             int cv0, int jac0, double* cvv, Jac J) {
    for (int i = 0; i < n; i++) {
        int s = off[i], e = off[i + 1], na = e - s;
        R sum = 0;
        std::vector<V3<R>> dr(na);
        for (int j = s; j < e; j++) {
            V3<R> p = P<R>(pos, atoms[j]);
            V3<R> d{p.x - (R)ref[3 * j], p.y - (R)ref[3 * j + 1], p.z - (R)ref[3 * j + 2]};
            sum += dot(d, d);
            dr[j - s] = d;
        }
        sum /= (R)na;
        R rmsd = std::sqrt(sum);
        R inv = rmsd > (R)1e-10 ? (R)1 / rmsd : (R)0;
        cvv[cv0 + i] = (double)rmsd;
        R scale = inv / (R)na;
        for (int j = s; j < e; j++) {
            V3<R> d = dr[j - s];
            J.set(jac0 + j, atoms[j], jstore<R>(d.x * scale), jstore<R>(d.y * scale), jstore<R>(d.z * scale), cv0 + i);
        }
    }
}

// Optimal-superposition (Kabsch) RMSD via the quaternion 4x4 eigenproblem in FP64.
// No reference counterpart (the reference RMSD is no-fit only); this is the
// independent FP64 definition the product's Kabsch extension is checked against.
// Jacobian: (1/(N*rmsd)) * (x_i - xc - R^T (y_i - yc)), rotation held fixed
// (exact at the optimum by the envelope theorem).
void jacobi4(double A[4][4], double V[4][4], double w[4]) {
    for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) V[i][j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 64; sweep++) {
        double off = 0;
        for (int p = 0; p < 4; p++) for (int q = p + 1; q < 4; q++) off += A[p][q] * A[p][q];
        if (off < 1e-30) break;
        for (int p = 0; p < 4; p++) for (int q = p + 1; q < 4; q++) {
            if (std::fabs(A[p][q]) < 1e-300) continue;
            double th = (A[q][q] - A[p][p]) / (2 * A[p][q]);
            double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1));
            double c = 1 / std::sqrt(t * t + 1), s = t * c;
            for (int k = 0; k < 4; k++) {
                double akp = A[k][p], akq = A[k][q];
                A[k][p] = c * akp - s * akq; A[k][q] = s * akp + c * akq;
            }
            for (int k = 0; k < 4; k++) {
                double apk = A[p][k], aqk = A[q][k];
                A[p][k] = c * apk - s * aqk; A[q][k] = s * apk + c * aqk;
            }
            for (int k = 0; k < 4; k++) {
                double vkp = V[k][p], vkq = V[k][q];
                V[k][p] = c * vkp - s * vkq; V[k][q] = s * vkp + c * vkq;
            }
        }
    }
    for (int i = 0; i < 4; i++) w[i] = A[i][i];
}

void cv_rmsd_kabsch_f64(const double* pos, const int* atoms, const float* ref, int na,
                        double* value, double* grad /* 3*na */) {
    double xc[3] = {0, 0, 0}, yc[3] = {0, 0, 0};
    for (int j = 0; j < na; j++) for (int k = 0; k < 3; k++) {
        xc[k] += pos[3 * atoms[j] + k]; yc[k] += (double)ref[3 * j + k];
    }
    for (int k = 0; k < 3; k++) { xc[k] /= na; yc[k] /= na; }
    double Rm[3][3] = {{0}}, G = 0;
    for (int j = 0; j < na; j++) {
        double x[3], y[3];
        for (int k = 0; k < 3; k++) { x[k] = pos[3 * atoms[j] + k] - xc[k]; y[k] = (double)ref[3 * j + k] - yc[k]; }
        for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) Rm[a][b] += x[a] * y[b];
        G += x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + y[0] * y[0] + y[1] * y[1] + y[2] * y[2];
    }
    double F[4][4] = {
        {Rm[0][0] + Rm[1][1] + Rm[2][2], Rm[1][2] - Rm[2][1], Rm[2][0] - Rm[0][2], Rm[0][1] - Rm[1][0]},
        {Rm[1][2] - Rm[2][1], Rm[0][0] - Rm[1][1] - Rm[2][2], Rm[0][1] + Rm[1][0], Rm[0][2] + Rm[2][0]},
        {Rm[2][0] - Rm[0][2], Rm[0][1] + Rm[1][0], -Rm[0][0] + Rm[1][1] - Rm[2][2], Rm[1][2] + Rm[2][1]},
        {Rm[0][1] - Rm[1][0], Rm[0][2] + Rm[2][0], Rm[1][2] + Rm[2][1], -Rm[0][0] - Rm[1][1] + Rm[2][2]}};
    double V[4][4], w[4];
    jacobi4(F, V, w);
    int im = 0;
    for (int i = 1; i < 4; i++) if (w[i] > w[im]) im = i;
    double q0 = V[0][im], q1 = V[1][im], q2 = V[2][im], q3 = V[3][im];
    // With the correlation matrix Rm = sum x y^T, the top eigenvector q is the
    // rotation that takes x onto y; its transpose takes y (reference) onto x:
    // x ~ Rot * y with Rot = R(q)^T.
    double Rot[3][3] = {
        {q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3, 2 * (q1 * q2 + q0 * q3), 2 * (q1 * q3 - q0 * q2)},
        {2 * (q1 * q2 - q0 * q3), q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3, 2 * (q2 * q3 + q0 * q1)},
        {2 * (q1 * q3 + q0 * q2), 2 * (q2 * q3 - q0 * q1), q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3}};
    double msd = std::max(0.0, (G - 2 * w[im]) / na);
    double rmsd = std::sqrt(msd);
    *value = rmsd;
    double sc = rmsd > 1e-10 ? 1.0 / (na * rmsd) : 0.0;
    for (int j = 0; j < na; j++) {
        double x[3], y[3], ry[3];
        for (int k = 0; k < 3; k++) { x[k] = pos[3 * atoms[j] + k] - xc[k]; y[k] = (double)ref[3 * j + k] - yc[k]; }
        for (int a = 0; a < 3; a++) ry[a] = Rot[a][0] * y[0] + Rot[a][1] * y[1] + Rot[a][2] * y[2];
        for (int k = 0; k < 3; k++) grad[3 * j + k] = sc * (x[k] - ry[k]);
    }
}

// Path CV (s, z) over N frames of M atoms: CommonGluedKernels.cpp:667-794.
// Frames are 1-indexed in s; the reference caches frame weights as float.
template <class R>
void cv_path(const double* pos, const int* off, const int* atoms, const int* refOff,
             const float* refPos, const float* prm, int n, int cv0, int jac0, double* cvv, Jac J) {
    for (int i = 0; i < n; i++) {
        int s0 = off[i], M = off[i + 1] - s0, rb = refOff[i];
        int N = (int)prm[2 * i + 1];
        R lam = (R)prm[2 * i];
        std::vector<R> w(N);
        R S = 0, sn = 0;
        for (int f = 0; f < N; f++) {
            R m2 = 0;
            for (int j = 0; j < M; j++) {
                V3<R> p = P<R>(pos, atoms[s0 + j]);
                int ri = 3 * (rb + f * M + j);
                R dx = p.x - (R)refPos[ri], dy = p.y - (R)refPos[ri + 1], dz = p.z - (R)refPos[ri + 2];
                m2 += dx * dx + dy * dy + dz * dz;
            }
            m2 /= (R)M;
            R wf = std::exp(-lam * m2);
            w[f] = std::is_same<R, float>::value ? (R)(float)wf : wf;
            S += wf;
            sn += (R)(f + 1) * wf;
        }
        R iS = S > (R)1e-300 ? (R)1 / S : (R)0;
        R s = sn * iS;
        R z = S > (R)1e-300 ? -std::log(S) / lam : (R)0;
        cvv[cv0 + 2 * i] = (double)s;
        cvv[cv0 + 2 * i + 1] = (double)z;
        R scS = (R)-2 * lam / ((R)M * S), scZ = (R)2 / ((R)M * S);
        for (int j = 0; j < M; j++) {
            int a = atoms[s0 + j];
            V3<R> p = P<R>(pos, a);
            R sx = 0, sy = 0, sz = 0, zx = 0, zy = 0, zz = 0;
            for (int f = 0; f < N; f++) {
                int ri = 3 * (rb + f * M + j);
                R dx = p.x - (R)refPos[ri], dy = p.y - (R)refPos[ri + 1], dz = p.z - (R)refPos[ri + 2];
                R wf = w[f], fs = ((R)(f + 1) - s) * wf;
                sx += fs * dx; sy += fs * dy; sz += fs * dz;
                zx += wf * dx; zy += wf * dy; zz += wf * dz;
            }
            J.set(jac0 + 2 * (s0 + j), a, jstore<R>(scS * sx), jstore<R>(scS * sy), jstore<R>(scS * sz), cv0 + 2 * i);
            J.set(jac0 + 2 * (s0 + j) + 1, a, jstore<R>(scZ * zx), jstore<R>(scZ * zy), jstore<R>(scZ * zz), cv0 + 2 * i + 1);
        }
    }
}

template <class R> inline R ipow(R x, int n) { R r = 1; for (int i = 0; i < n; i++) r *= x; return r; }

// Contact map: CommonGluedKernels.cpp:1236-1323. Per pair [r0, n, m, w] (float),
// integer exponents, |den| < 1e-8 -> s = n/m.
template <class R>
void cv_contact_map(const double* pos, const int* off, const int* pairs, const float* prm, int n,
                    int cv0, int jac0, const double* box9, int periodic, double* cvv, Jac J) {
    Box<R> box(box9);
    for (int i = 0; i < n; i++) {
        R v = 0;
        for (int p = off[i]; p < off[i + 1]; p++) {
            int a = pairs[2 * p], b = pairs[2 * p + 1];
            R r0 = (R)prm[4 * p], w = (R)prm[4 * p + 3];
            int nn = (int)prm[4 * p + 1], mm = (int)prm[4 * p + 2];
            V3<R> d = sub(P<R>(pos, b), P<R>(pos, a));
            if (periodic) d = box.image(d);
            R dist = std::sqrt(dot(d, d));
            R idist = dist > (R)1e-10 ? (R)1 / dist : (R)0;
            R ir0 = (R)1 / r0, x = dist * ir0;
            R xn = ipow(x, nn), xm = ipow(x, mm), num = (R)1 - xn, den = (R)1 - xm;
            R s, dsdd;
            if (std::fabs(den) < (R)1e-8) { s = (R)nn / (R)mm; dsdd = 0; }
            else {
                s = num / den;
                R dxn = nn > 0 ? (R)nn * ipow(x, nn - 1) : (R)0;
                R dxm = mm > 0 ? (R)mm * ipow(x, mm - 1) : (R)0;
                dsdd = ((-dxn * den + dxm * num) / (den * den)) * ir0;
            }
            v += w * s;
            R co = w * dsdd * idist;
            J.set(jac0 + 2 * p, a, jstore<R>(-co * d.x), jstore<R>(-co * d.y), jstore<R>(-co * d.z), cv0 + i);
            J.set(jac0 + 2 * p + 1, b, jstore<R>(co * d.x), jstore<R>(co * d.y), jstore<R>(co * d.z), cv0 + i);
        }
        cvv[cv0 + i] = (double)v;
    }
}

// PCA projection, FP64 accumulator: CommonGluedKernels.cpp:1633-1681.
template <class R>
void cv_pca(const double* pos, const int* off, const int* atoms, const float* ref, const float* ev,
            int n, int cv0, int jac0, double* cvv, Jac J) {
    for (int i = 0; i < n; i++) {
        double acc = 0;
        for (int j = off[i]; j < off[i + 1]; j++) {
            V3<R> p = P<R>(pos, atoms[j]);
            R dx = p.x - (R)ref[3 * j], dy = p.y - (R)ref[3 * j + 1], dz = p.z - (R)ref[3 * j + 2];
            acc += (double)(dx * (R)ev[3 * j] + dy * (R)ev[3 * j + 1] + dz * (R)ev[3 * j + 2]);
        }
        cvv[cv0 + i] = acc;
        for (int j = off[i]; j < off[i + 1]; j++)
            J.set(jac0 + j, atoms[j], (double)ev[3 * j], (double)ev[3 * j + 1], (double)ev[3 * j + 2], cv0 + i);
    }
}

}  // namespace

// ===================================================================== C ABI
extern "C" {

#define ORC_JAC int* ja, double* jx, double* jy, double* jz, int* jc
#define ORC_J Jac{ja, jx, jy, jz, jc}

#define ORC_BOTH(name, sig, call)                                   \
    void orc_##name##_f32 sig { name<float> call; }                  \
    void orc_##name##_f64 sig { name<double> call; }

ORC_BOTH(cv_distance, (const double* pos, const int* a, int n, int cv0, int jac0, const double* box, int per, double* cvv, ORC_JAC),
         (pos, a, n, cv0, jac0, box, per, cvv, ORC_J))
ORC_BOTH(cv_angle, (const double* pos, const int* a, int n, int cv0, int jac0, const double* box, int per, double* cvv, ORC_JAC),
         (pos, a, n, cv0, jac0, box, per, cvv, ORC_J))
ORC_BOTH(cv_dihedral, (const double* pos, const int* a, int n, int cv0, int jac0, const double* box, int per, double* cvv, ORC_JAC),
         (pos, a, n, cv0, jac0, box, per, cvv, ORC_J))
ORC_BOTH(cv_com_distance, (const double* pos, const int* off, const int* at, const float* m, const float* tm, int n, int cv0, int jac0, const double* box, int per, double* cvv, ORC_JAC),
         (pos, off, at, m, tm, n, cv0, jac0, box, per, cvv, ORC_J))
ORC_BOTH(cv_gyration, (const double* pos, const int* off, const int* at, const float* m, const float* tm, int n, int cv0, int jac0, const double* box, int per, double* cvv, ORC_JAC),
         (pos, off, at, m, tm, n, cv0, jac0, box, per, cvv, ORC_J))
ORC_BOTH(cv_coordination, (const double* pos, const int* off, const int* at, const float* prm, int n, int cv0, int jac0, const double* box, int per, double rc, double* cvv, ORC_JAC),
         (pos, off, at, prm, n, cv0, jac0, box, per, rc, cvv, ORC_J))
ORC_BOTH(cv_rmsd, (const double* pos, const int* off, const int* at, const float* ref, int n, int cv0, int jac0, double* cvv, ORC_JAC),
         (pos, off, at, ref, n, cv0, jac0, cvv, ORC_J))
ORC_BOTH(cv_path, (const double* pos, const int* off, const int* at, const int* roff, const float* ref, const float* prm, int n, int cv0, int jac0, double* cvv, ORC_JAC),
         (pos, off, at, roff, ref, prm, n, cv0, jac0, cvv, ORC_J))
ORC_BOTH(cv_contact_map, (const double* pos, const int* off, const int* pr, const float* prm, int n, int cv0, int jac0, const double* box, int per, double* cvv, ORC_JAC),
         (pos, off, pr, prm, n, cv0, jac0, box, per, cvv, ORC_J))
ORC_BOTH(cv_pca, (const double* pos, const int* off, const int* at, const float* ref, const float* ev, int n, int cv0, int jac0, double* cvv, ORC_JAC),
         (pos, off, at, ref, ev, n, cv0, jac0, cvv, ORC_J))

void orc_cv_rmsd_kabsch(const double* pos, const int* atoms, const float* ref, int na, double* value, double* grad) {
    cv_rmsd_kabsch_f64(pos, atoms, ref, na, value, grad);
}

// Chain-rule scatter into a 2^32 fixed-point, field-major int64 force buffer:
// CommonGluedKernels.cpp:2430-2456. The double product is truncated toward zero
// by the (long long) conversion, as in the reference.
void orc_scatter(const double* dUdCV, const int* ja, const double* jx, const double* jy, const double* jz,
                 const int* jc, int rows, long long* force, int padded) {
    const double S = 4294967296.0;
    for (int j = 0; j < rows; j++) {
        double g = dUdCV[jc[j]];
        long long fx = (long long)(-(g * jx[j]) * S);
        long long fy = (long long)(-(g * jy[j]) * S);
        long long fz = (long long)(-(g * jz[j]) * S);
        uint64_t* f = reinterpret_cast<uint64_t*>(force);
        f[ja[j]] += (uint64_t)fx;
        f[ja[j] + padded] += (uint64_t)fy;
        f[ja[j] + 2 * padded] += (uint64_t)fz;
    }
}

// Harmonic restraint with optional 2*pi wrap; (k, s0) stored as float:
// CommonGluedKernels.cpp:2513-2540 and CommonBiasKernels.cpp:115-125.
double orc_harmonic(const double* cvv, const int* idx, const float* prm, int d, int periodic, double* grad) {
    const double TWO_PI = 6.283185307179586;
    double V = 0;
    for (int i = 0; i < d; i++) {
        double s = cvv[idx[i]], k = (double)prm[2 * i], s0 = (double)prm[2 * i + 1];
        double ds = s - s0;
        if (periodic) ds -= TWO_PI * std::round(ds / TWO_PI);
        V += 0.5 * k * ds * ds;
        grad[idx[i]] += k * ds;
    }
    return V;
}

// MetaD grid: multilinear interpolation over 2^D corners with periodic wrap or
// clamping: CommonGluedKernels.cpp:3574-3636. Column-major grid.
double orc_metad_eval(const double* cvv, const int* idx, int D, const double* grid, const double* origin,
                      const double* invSp, const int* npts, const int* stride, const int* per, double* grad) {
    int lo[3], hi[3]; double al[3];
    for (int d = 0; d < D; d++) {
        double fr = (cvv[idx[d]] - origin[d]) * invSp[d];
        int N = npts[d];
        if (N <= 1) { lo[d] = hi[d] = 0; al[d] = 0; }
        else if (per[d]) {
            fr = fr - std::floor(fr / (double)N) * (double)N;
            if (fr < 0.0) fr += N;
            lo[d] = (int)fr;
            if (lo[d] >= N) lo[d] = N - 1;
            al[d] = fr - lo[d];
            hi[d] = (lo[d] + 1) % N;
        } else {
            if (fr < 0.0) fr = 0.0;
            if (fr > (double)(N - 1)) fr = (double)(N - 1);
            lo[d] = (int)fr;
            if (lo[d] >= N - 1) lo[d] = N - 2;
            al[d] = fr - lo[d];
            hi[d] = lo[d] + 1;
        }
    }
    double V = 0, dV[3] = {0, 0, 0};
    for (int c = 0; c < (1 << D); c++) {
        int flat = 0;
        for (int d = 0; d < D; d++) flat += (((c >> d) & 1) ? hi[d] : lo[d]) * stride[d];
        double val = grid[flat], w = 1;
        for (int d = 0; d < D; d++) w *= ((c >> d) & 1) ? al[d] : (1.0 - al[d]);
        V += w * val;
        for (int d = 0; d < D; d++) {
            double sg = ((c >> d) & 1) ? 1.0 : -1.0, wo = 1;
            for (int e = 0; e < D; e++) if (e != d) wo *= ((c >> e) & 1) ? al[e] : (1.0 - al[e]);
            dV[d] += sg * wo * val;
        }
    }
    for (int d = 0; d < D; d++) grad[idx[d]] += dV[d] * invSp[d];
    return V;
}

// MetaD Gaussian deposit on the whole grid, truncated at exponent > 8:
// CommonGluedKernels.cpp:3645-3680; height h0*exp(-V*heightInvFactor) from the
// same bias's last V (CommonBiasKernels.cpp:256).
void orc_metad_deposit(double* grid, int D, int total, const double* origin, const double* invSp,
                       const int* npts, const int* stride, const int* per, const double* center,
                       const double* sigma, double Vlast, double h0, double hif) {
    double h = hif > 0.0 ? h0 * std::exp(-Vlast * hif) : h0;
    for (int idx = 0; idx < total; idx++) {
        double ex = 0;
        for (int d = 0; d < D; d++) {
            int bi = (idx / stride[d]) % npts[d];
            double p = origin[d] + (double)bi / invSp[d];
            double dc = p - center[d];
            if (per[d]) { double L = (double)npts[d] / invSp[d]; dc -= std::round(dc / L) * L; }
            ex += dc * dc / (2.0 * sigma[d] * sigma[d]);
        }
        if (ex <= 8.0) grid[idx] += h * std::exp(-ex);
    }
}

// PBMETAD: N 1-D sub-grids (concatenated, sub-grid d at goff[d]) over the CVs
// idx[d], each linearly interpolated with periodic wrap or clamping
// (CommonGluedKernels.cpp:3698-3734), combined by log-sum-exp
// E = -kT (ln sum_d exp((Vmin - V_d)/kT) - ln N) + Vmin with dE/ds_d = w_d dV_d/ds_d,
// w_d the softmax weights (:3736-3763). V_d and w_d are returned for the deposit.
double orc_pbmetad_eval(const double* cvv, const int* idx, int N, const double* grid, const int* goff,
                        const double* origin, const double* invSp, const int* npts, const int* per, double kT,
                        double* grad, double* Vout, double* Wout) {
    double G[8];
    for (int d = 0; d < N; d++) {
        const double* g = grid + goff[d];
        const int n = npts[d];
        double fr = (cvv[idx[d]] - origin[d]) * invSp[d];
        int lo, hi;
        if (per[d]) {
            fr = fr - std::floor(fr / (double)n) * (double)n;
            if (fr < 0.0) fr += (double)n;
            lo = (int)fr;
            if (lo >= n) lo = n - 1;
            hi = (lo + 1) % n;
        } else {
            if (fr < 0.0) fr = 0.0;
            if (fr > (double)(n - 1)) fr = (double)(n - 1);
            lo = (int)fr;
            if (lo >= n - 1) lo = n - 2;
            hi = lo + 1;
        }
        const double al = fr - lo;
        Vout[d] = g[lo] * (1.0 - al) + g[hi] * al;
        G[d] = (g[hi] - g[lo]) * invSp[d];
    }
    double vmin = Vout[0];
    for (int d = 1; d < N; d++)
        if (Vout[d] < vmin) vmin = Vout[d];
    double sum = 0.0;
    for (int d = 0; d < N; d++) sum += std::exp((vmin - Vout[d]) / kT);
    for (int d = 0; d < N; d++) {
        Wout[d] = std::exp((vmin - Vout[d]) / kT) / sum;
        grad[idx[d]] += Wout[d] * G[d];
    }
    return -kT * (std::log(sum) - std::log((double)N)) + vmin;
}

// PBMETAD deposit (CommonGluedKernels.cpp:3765-3797, pace gate :5147-5155): each
// sub-grid d gets a 1-D Gaussian at its CV value with height w_d h0 exp(-V_d hif)
// (w_d h0 when hif = 0), V_d and w_d from the last evaluation, exponent <= 8.
void orc_pbmetad_deposit(double* grid, const int* goff, int N, const double* origin, const double* invSp,
                         const int* npts, const int* per, const double* cvv, const int* idx, const double* sigma,
                         const double* V, const double* W, double h0, double hif) {
    for (int d = 0; d < N; d++) {
        const double height = hif > 0.0 ? W[d] * h0 * std::exp(-V[d] * hif) : W[d] * h0;
        double* g = grid + goff[d];
        for (int i = 0; i < npts[d]; i++) {
            double dc = origin[d] + (double)i / invSp[d] - cvv[idx[d]];
            if (per[d]) {
                const double L = (double)npts[d] / invSp[d];
                dc -= std::round(dc / L) * L;
            }
            const double ex = dc * dc / (2.0 * sigma[d] * sigma[d]);
            if (ex <= 8.0) g[i] += height * std::exp(-ex);
        }
    }
}

// Direct hill sum V(s) = sum_k h_k exp(-sum_d dc^2 / (2 sigma_d^2)), exponent > 8
// truncated like the grid deposit, periodic wrap with period L_d (L_d <= 0 means
// non-periodic). No reference counterpart (the reference MetaD is grid-only).
double orc_hills_eval(const double* s, int D, const double* centers, const double* heights, int K,
                      const double* sigma, const double* period, double* dVds) {
    double V = 0;
    for (int d = 0; d < D; d++) dVds[d] = 0;
    for (int k = 0; k < K; k++) {
        double ex = 0, dc[8];
        for (int d = 0; d < D; d++) {
            double x = s[d] - centers[k * D + d];
            if (period[d] > 0) x -= std::round(x / period[d]) * period[d];
            dc[d] = x;
            ex += x * x / (2.0 * sigma[d] * sigma[d]);
        }
        if (ex > 8.0) continue;
        double g = heights[k] * std::exp(-ex);
        V += g;
        for (int d = 0; d < D; d++) dVds[d] += -g * dc[d] / (sigma[d] * sigma[d]);
    }
    return V;
}

// OPES kernel-sum bias: CommonGluedKernels.cpp:2642-2723. Returns V; adds dV/ds
// into grad[idx[d]].
double orc_opes_eval(const double* cvv, const int* idx, int D, const double* centers, const double* sigmas,
                     const double* logW, int K, double invGF, double kT, double sumUprob, double cutoff2,
                     double eps, double barrier, double* grad) {
    if (K == 0) return -barrier;
    double kfloor = std::exp(-0.5 * cutoff2), prob = 0, acc[16] = {0};
    for (int k = 0; k < K; k++) {
        double n2 = 0, dc[16], sg[16];
        for (int d = 0; d < D; d++) {
            dc[d] = cvv[idx[d]] - centers[k * D + d];
            sg[d] = sigmas[k * D + d];
            n2 += dc[d] * dc[d] / (sg[d] * sg[d]);
        }
        if (!(n2 < cutoff2)) continue;
        double G = std::exp(-0.5 * n2), kern = G - kfloor;
        if (kern <= 0.0) continue;
        double h = std::exp(logW[k]);
        if (!(h > 0.0 && h < 1e308)) continue;
        prob += h * kern;
        for (int d = 0; d < D; d++) acc[d] += h * G * (-dc[d] / (sg[d] * sg[d]));
    }
    double pz = sumUprob > 0.0 ? prob * (double)K / sumUprob : 0.0;
    if (!(pz >= 0.0)) pz = 0.0;
    double arg = pz + eps;
    double V = invGF * kT * std::log(arg > 1e-30 ? arg : 1e-30);
    if (prob > 0.0) {
        double f = invGF * kT * (pz / (pz + eps)) / prob;
        for (int d = 0; d < D; d++) grad[idx[d]] += f * acc[d];
    }
    return V;
}

// OPES deposit with Silverman bandwidth, compression (merge) decision and the
// incremental / full sum_uprob update: CommonGluedKernels.cpp:2752-3003.
// State vector layout (double): st[0]=sum_uprob, st[1]=sumWeights, st[2]=sum_w,
// st[3]=sum_w2; ist[0]=numKernels, ist[1]=nSamples, ist[2]=stepCount,
// ist[3]=numAllocated. Returns the merge index (>=0), -1 for an append, -2 when
// the deposit was skipped (adaptive warm-up) and -3 when the table is full.
// Transcendentals use the deterministic gd_exp/gd_log/gd_pow shared with the
// device code so that decisions can be compared bit for bit.
int orc_opes_deposit_ex(const double* cvv, const int* idx, int D, double* runMean, double* runM2,
                        const double* sigma0, double sigmaMin, double* centers, double* sigmas, double* logW,
                        double* st, int* ist, int variant, int adaptiveStride, double Vlast, double invKT,
                        double cutoff2, int maxKernels, double gamma, int skipPairSum);

int orc_opes_deposit(const double* cvv, const int* idx, int D, double* runMean, double* runM2,
                     const double* sigma0, double sigmaMin, double* centers, double* sigmas, double* logW,
                     double* st, int* ist, int variant, int adaptiveStride, double Vlast, double invKT,
                     double cutoff2, int maxKernels, double gamma) {
    return orc_opes_deposit_ex(cvv, idx, D, runMean, runM2, sigma0, sigmaMin, centers, sigmas, logW, st, ist,
                               variant, adaptiveStride, Vlast, invKT, cutoff2, maxKernels, gamma, 0);
}

// skipPairSum != 0 leaves sum_uprob untouched (decision replays: the sum feeds
// only the bias value, never a merge decision).
int orc_opes_deposit_ex(const double* cvv, const int* idx, int D, double* runMean, double* runM2,
                        const double* sigma0, double sigmaMin, double* centers, double* sigmas, double* logW,
                        double* st, int* ist, int variant, int adaptiveStride, double Vlast, double invKT,
                        double cutoff2, int maxKernels, double gamma, int skipPairSum) {
    using namespace glued_dmath;
    if (adaptiveStride > 0 && ist[1] < adaptiveStride) return -2;
    int nB = ist[0];
    if (variant != 1 && adaptiveStride == 0) ist[1]++;
    int n = ist[1];
    double c[16], sg[16];
    for (int d = 0; d < D; d++) c[d] = cvv[idx[d]];
    double VkT = Vlast * invKT, lwRaw, hRaw;
    if (variant == 2) { lwRaw = 0.0; hRaw = 1.0; } else { lwRaw = VkT; hRaw = gd_exp(VkT); }
    st[2] += hRaw;
    st[3] += hRaw * hRaw;
    ist[2]++;
    double sw = st[2], sw2 = st[3];
    double neff = (1.0 + sw) * (1.0 + sw) / (1.0 + sw2);
    double size = variant == 2 ? (double)ist[2] : neff;
    for (int d = 0; d < D; d++) {
        double s;
        if (variant == 1) s = sigma0[d];
        else if (adaptiveStride > 0) {
            double factor = variant == 2 ? 1.0 : gamma;
            double var = n > 1 ? runM2[d] / factor / (double)(n - 1) : 0.0;
            s = var > 0.0 ? std::sqrt(var) : 1.0;
            if (s < sigmaMin) s = sigmaMin;
        } else {
            double resc = gd_pow(size * (D + 2) / 4.0, -1.0 / (D + 4.0));
            s = sigma0[d] * resc;
            if (s < sigmaMin) s = sigmaMin;
        }
        sg[d] = s;
    }
    double lwNew = lwRaw;
    if (variant != 1 && adaptiveStride == 0)
        for (int d = 0; d < D; d++) lwNew += gd_log(sigma0[d] / sg[d]);
    double hNew = gd_exp(lwNew);
    int mk = -1; double minN2 = 1.0;
    for (int kp = 0; kp < nB; kp++) {
        double n2 = 0; bool over = false;
        for (int d = 0; d < D; d++) {
            double x = (c[d] - centers[kp * D + d]) / sigmas[kp * D + d];
            n2 += x * x;
            if (n2 >= minN2) { over = true; break; }
        }
        if (!over) { minN2 = n2; mk = kp; }
    }
    int nA, ret;
    if (mk >= 0) {
        double lwo = logW[mk], ho = gd_exp(lwo), ht = ho + hNew;
        double lmax = lwo > lwNew ? lwo : lwNew, lmin = lwo < lwNew ? lwo : lwNew;
        double lwm = lmax + gd_log1p(gd_exp(lmin - lmax));
        double f1 = ho / ht, f2 = hNew / ht;
        for (int d = 0; d < D; d++) {
            double c1 = centers[mk * D + d], s1 = sigmas[mk * D + d], c2 = c[d], s2 = sg[d];
            double cm = f1 * c1 + f2 * c2;
            double ss = f1 * (s1 * s1 + c1 * c1) + f2 * (s2 * s2 + c2 * c2) - cm * cm;
            if (ss < 0.0) ss = 0.0;
            double sm = std::sqrt(ss);
            if (sm < sigmaMin) sm = sigmaMin;
            centers[mk * D + d] = cm; sigmas[mk * D + d] = sm;
        }
        logW[mk] = lwm;
        nA = nB; ret = mk;
    } else {
        int k = ist[3]++;
        if (k < maxKernels) {
            for (int d = 0; d < D; d++) { centers[k * D + d] = c[d]; sigmas[k * D + d] = sg[d]; }
            logW[k] = lwNew;
            ist[0]++;
            nA = nB + 1; ret = -1;
        } else { ist[3]--; nA = nB; ret = -3; }
    }
    st[1] += hRaw;
    double eps = gd_exp(-0.5 * cutoff2);
    if (skipPairSum) return ret;
    if (mk < 0 && nA > nB) {
        double delta = hNew * (1.0 - eps);
        for (int j = 0; j < nB; j++) {
            double n2 = 0; bool skip = false;
            for (int d = 0; d < D; d++) {
                double dc = centers[j * D + d] - c[d];
                n2 += dc * dc / (sg[d] * sg[d]);
                if (n2 >= cutoff2) { skip = true; break; }
            }
            if (!skip) delta += hNew * (gd_exp(-0.5 * n2) - eps);
        }
        for (int kp = 0; kp < nB; kp++) {
            double n2 = 0; bool skip = false;
            for (int d = 0; d < D; d++) {
                double dc = c[d] - centers[kp * D + d], s = sigmas[kp * D + d];
                n2 += dc * dc / (s * s);
                if (n2 >= cutoff2) { skip = true; break; }
            }
            if (!skip) delta += gd_exp(logW[kp]) * (gd_exp(-0.5 * n2) - eps);
        }
        st[0] += delta;
    } else {
        double su = 0;
        for (int j = 0; j < nA; j++)
            for (int kp = 0; kp < nA; kp++) {
                double n2 = 0; bool skip = false;
                for (int d = 0; d < D; d++) {
                    double dc = centers[j * D + d] - centers[kp * D + d], s = sigmas[kp * D + d];
                    n2 += dc * dc / (s * s);
                    if (n2 >= cutoff2) { skip = true; break; }
                }
                if (skip) continue;
                su += gd_exp(logW[kp]) * (gd_exp(-0.5 * n2) - eps);
            }
        st[0] = su;
    }
    return ret;
}

// Per-step Welford accumulation for fully adaptive sigma:
// CommonGluedKernels.cpp:3009-3027.
void orc_opes_welford(const double* cvv, const int* idx, int D, double* mean, double* m2, int* nSamples) {
    int n = ++nSamples[0];
    for (int d = 0; d < D; d++) {
        double x = cvv[idx[d]], dl = x - mean[d];
        mean[d] += dl / n;
        m2[d] += dl * (x - mean[d]);
    }
}

}  // extern "C"
