// goqu's parameterized gate matrices and their derivatives (see params.hpp).
#include "params.hpp"

#include <cmath>

namespace gq {

namespace {

Z ex(double x) { return Z{std::cos(x), std::sin(x)}; }  // cmplx.Exp(complex(0, x))
Z scl(Z a, double s) { return Z{a.re * s, a.im * s}; }
Z neg(Z a) { return Z{-a.re, -a.im}; }
Z iz(Z a) { return Z{-a.im, a.re}; }  // i * a
const Z kZero{0.0, 0.0}, kOne{1.0, 0.0};

// Families whose derivative is exp(-i t/2 G)' = U(t + pi) / 2 (G^2 = I).
bool shift_family(int f) {
    return f == GQ_PG_RX || f == GQ_PG_RY || f == GQ_PG_RZ || f == GQ_PG_RXX || f == GQ_PG_RYY || f == GQ_PG_RZZ;
}

int angle_count(int f) {
    switch (f) {
        case GQ_PG_U3: case GQ_PG_ROT: return 3;
        case GQ_PG_U2: case GQ_PG_FSIM: return 2;
        default: return 1;
    }
}

}  // namespace

bool param_gate_matrix(int f, const double* a, int na, std::vector<Z>& m) {
    if (na != angle_count(f)) return false;
    const double t = a[0];
    switch (f) {
        case GQ_PG_RX: {  // parameterized.go RX
            const double c = std::cos(t / 2), s = std::sin(t / 2);
            m = {Z{c, 0}, Z{0, -s}, Z{0, -s}, Z{c, 0}};
            return true;
        }
        case GQ_PG_RY: {
            const double c = std::cos(t / 2), s = std::sin(t / 2);
            m = {Z{c, 0}, Z{-s, 0}, Z{s, 0}, Z{c, 0}};
            return true;
        }
        case GQ_PG_RZ:
            m = {ex(-t / 2), kZero, kZero, ex(t / 2)};
            return true;
        case GQ_PG_PHASE:
        case GQ_PG_U1:
            m = {kOne, kZero, kZero, ex(t)};
            return true;
        case GQ_PG_GLOBAL_PHASE:
            m = {ex(t), kZero, kZero, ex(t)};
            return true;
        case GQ_PG_U3: {
            const double c = std::cos(t / 2), s = std::sin(t / 2);
            m = {Z{c, 0}, neg(scl(ex(a[2]), s)), scl(ex(a[1]), s), scl(ex(a[1] + a[2]), c)};
            return true;
        }
        case GQ_PG_U2: {
            const double s = M_SQRT1_2;
            m = {Z{s, 0}, neg(scl(ex(a[1]), s)), scl(ex(a[0]), s), scl(ex(a[0] + a[1]), s)};
            return true;
        }
        case GQ_PG_ROT: {  // (phi, theta, omega)
            const double c = std::cos(a[1] / 2), s = std::sin(a[1] / 2);
            const Z ipo = ex((a[0] + a[2]) / 2), imo = ex((a[0] - a[2]) / 2);
            m = {scl(Z{ipo.re, -ipo.im}, c), neg(scl(Z{imo.re, -imo.im}, s)), scl(imo, s), scl(ipo, c)};
            return true;
        }
        case GQ_PG_CP:
            m.assign(16, kZero);
            m[0] = m[5] = m[10] = kOne;
            m[15] = ex(t);
            return true;
        case GQ_PG_RXX: {
            const double c = std::cos(t / 2), s = std::sin(t / 2);
            m.assign(16, kZero);
            m[0] = m[5] = m[10] = m[15] = Z{c, 0};
            m[3] = m[6] = m[9] = m[12] = Z{0, -s};
            return true;
        }
        case GQ_PG_RYY: {
            const double c = std::cos(t / 2), s = std::sin(t / 2);
            m.assign(16, kZero);
            m[0] = m[5] = m[10] = m[15] = Z{c, 0};
            m[3] = m[12] = Z{0, s};
            m[6] = m[9] = Z{0, -s};
            return true;
        }
        case GQ_PG_RZZ:
            m.assign(16, kZero);
            m[0] = m[15] = ex(-t / 2);
            m[5] = m[10] = ex(t / 2);
            return true;
        case GQ_PG_FSIM: {
            const double c = std::cos(t), s = std::sin(t);
            m.assign(16, kZero);
            m[0] = kOne;
            m[5] = m[10] = Z{c, 0};
            m[6] = m[9] = Z{0, -s};
            m[15] = ex(-a[1]);
            return true;
        }
        case GQ_PG_PSWAP:
            m.assign(16, kZero);
            m[0] = m[15] = kOne;
            m[6] = m[9] = ex(t);
            return true;
        default:
            return false;
    }
}

bool param_gate_dmatrix(int f, const double* a, int na, int k, std::vector<Z>& dm) {
    if (na != angle_count(f) || k < 0 || k >= na) return false;
    std::vector<Z> u;
    if (shift_family(f)) {
        const double t = a[0] + M_PI;
        if (!param_gate_matrix(f, &t, 1, u)) return false;
        dm.resize(u.size());
        for (size_t i = 0; i < u.size(); ++i) dm[i] = scl(u[i], 0.5);
        return true;
    }
    if (!param_gate_matrix(f, a, na, u)) return false;
    dm.assign(u.size(), kZero);
    switch (f) {
        case GQ_PG_PHASE: case GQ_PG_U1: case GQ_PG_CP:  // i e^(i phi) on the last diagonal entry
            dm.back() = iz(u.back());
            return true;
        case GQ_PG_GLOBAL_PHASE:
            for (size_t i = 0; i < u.size(); ++i) dm[i] = iz(u[i]);
            return true;
        case GQ_PG_U3: {
            const double c = std::cos(a[0] / 2), s = std::sin(a[0] / 2);
            if (k == 0) {
                dm = {Z{-s / 2, 0}, neg(scl(ex(a[2]), c / 2)), scl(ex(a[1]), c / 2), scl(ex(a[1] + a[2]), -s / 2)};
            } else if (k == 1) {
                dm = {kZero, kZero, iz(u[2]), iz(u[3])};
            } else {
                dm = {kZero, iz(u[1]), kZero, iz(u[3])};
            }
            return true;
        }
        case GQ_PG_U2:
            if (k == 0) dm = {kZero, kZero, iz(u[2]), iz(u[3])};
            else dm = {kZero, iz(u[1]), kZero, iz(u[3])};
            return true;
        case GQ_PG_ROT: {
            if (k == 1) {
                const double c = std::cos(a[1] / 2), s = std::sin(a[1] / 2);
                const Z ipo = ex((a[0] + a[2]) / 2), imo = ex((a[0] - a[2]) / 2);
                dm = {scl(Z{ipo.re, -ipo.im}, -s / 2), neg(scl(Z{imo.re, -imo.im}, c / 2)), scl(imo, c / 2),
                      scl(ipo, -s / 2)};
                return true;
            }
            // phi (k = 0): entries scale by -i/2, -i/2, i/2, i/2; omega (k = 2): -i/2, i/2, -i/2, i/2
            const double s0 = k == 0 ? -0.5 : -0.5, s1 = k == 0 ? -0.5 : 0.5, s2 = k == 0 ? 0.5 : -0.5, s3 = 0.5;
            dm = {scl(iz(u[0]), s0), scl(iz(u[1]), s1), scl(iz(u[2]), s2), scl(iz(u[3]), s3)};
            return true;
        }
        case GQ_PG_FSIM:
            if (k == 0) {
                const double c = std::cos(a[0]), s = std::sin(a[0]);
                dm[5] = dm[10] = Z{-s, 0};
                dm[6] = dm[9] = Z{0, -c};
            } else {
                dm[15] = neg(iz(u[15]));
            }
            return true;
        case GQ_PG_PSWAP:
            dm[6] = iz(u[6]);
            dm[9] = iz(u[9]);
            return true;
        default:
            return false;
    }
}

int bind_template(const gq_op* ops, size_t n_ops, const gq_param_gate* pg, size_t n_pg, const double* theta,
                  size_t n_params, BoundTemplate& out, std::string& err) {
    out.ops.assign(ops, ops + n_ops);
    out.store.clear();
    out.store.reserve(n_pg * 4);
    for (size_t g = 0; g < n_pg; ++g) {
        const gq_param_gate& p = pg[g];
        if (p.op_index < 0 || (size_t)p.op_index >= n_ops) {
            err = "parameterized gate " + std::to_string(g) + ": op index out of range";
            return GQ_EINVAL;
        }
        if (p.num_angles < 1 || p.num_angles > 3) {
            err = "parameterized gate " + std::to_string(g) + ": bad angle count";
            return GQ_EINVAL;
        }
        double ang[3];
        for (int k = 0; k < p.num_angles; ++k) {
            if (p.param[k] >= (int32_t)n_params) {
                err = "parameterized gate " + std::to_string(g) + ": parameter index out of range";
                return GQ_EINVAL;
            }
            ang[k] = p.scale[k] * (p.param[k] >= 0 ? theta[p.param[k]] : 0.0) + p.shift[k];
        }
        std::vector<Z> m;
        if (!param_gate_matrix(p.gate, ang, p.num_angles, m)) {
            err = "parameterized gate " + std::to_string(g) + ": unknown family or angle count";
            return GQ_EUNSUPPORTED;
        }
        gq_op& op = out.ops[p.op_index];
        out.store.push_back(std::move(m));
        op.matrix = (const double*)out.store.back().data();
        for (int s = 0; s < GQ_MAX_OP_PARAMS; ++s) {
            op.param_index[s] = -1;
            op.dmatrix[s] = nullptr;
        }
        int slots = 0;
        for (int k = 0; k < p.num_angles; ++k) {
            const int pi = p.param[k];
            if (pi < 0 || p.scale[k] == 0.0) continue;
            bool seen = false;
            for (int k2 = 0; k2 < k; ++k2) seen = seen || (p.param[k2] == pi && p.scale[k2] != 0.0);
            if (seen) continue;
            // chain rule over every angle of this gate that uses parameter pi
            std::vector<Z> total;
            for (int k2 = k; k2 < p.num_angles; ++k2) {
                if (p.param[k2] != pi || p.scale[k2] == 0.0) continue;
                std::vector<Z> d;
                param_gate_dmatrix(p.gate, ang, p.num_angles, k2, d);
                if (total.empty()) total.assign(d.size(), Z{0, 0});
                for (size_t i = 0; i < d.size(); ++i) {
                    total[i].re += p.scale[k2] * d[i].re;
                    total[i].im += p.scale[k2] * d[i].im;
                }
            }
            if (slots == GQ_MAX_OP_PARAMS) {
                err = "parameterized gate " + std::to_string(g) + ": more than three parameters";
                return GQ_EUNSUPPORTED;
            }
            out.store.push_back(std::move(total));
            op.param_index[slots] = pi;
            op.dmatrix[slots] = (const double*)out.store.back().data();
            ++slots;
        }
    }
    return GQ_OK;
}

}  // namespace gq
