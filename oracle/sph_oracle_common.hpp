// sph_oracle_common.hpp -- TEST INFRASTRUCTURE ONLY.
//
// The oracle is a CPU restatement of the reference's Taichi kernels for the per-step
// particle hot path (sigmaSPH v0.1.3).  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load it, always as the checker or the timed CPU baseline;
// the product path (sigmasph_b200) never links or calls it.
//
// Parity status: the reference's own Taichi run cannot execute on this machine
// (taichi is not installed and there is no network), so the restatement is pinned
// against (a) the reference's host-side float64 mirrors (tait_pressure_py,
// j2_radial_return_py, jc_radial_return_py), imported from the reference source to make
// the golden fixtures under tests/golden/, and (b) the known-answer values stated in the
// reference's comments (lambda plateau, lattice neighbour counts, hourglass kernel sum).
// The 3x3 symmetric eigensolver (ti.sym_eig in the reference) is third-party arithmetic
// that no shipped test pins; it is restated as a cyclic Jacobi solver and checked
// against numpy.linalg.eigh.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace orc {

template <class R> struct V3 {
    R a[3];
    V3() : a{R(0), R(0), R(0)} {}
    V3(R x, R y, R z) : a{x, y, z} {}
    R& operator[](int k) { return a[k]; }
    const R& operator[](int k) const { return a[k]; }
};
template <class R> inline V3<R> operator+(const V3<R>& p, const V3<R>& q) { return {p[0] + q[0], p[1] + q[1], p[2] + q[2]}; }
template <class R> inline V3<R> operator-(const V3<R>& p, const V3<R>& q) { return {p[0] - q[0], p[1] - q[1], p[2] - q[2]}; }
template <class R> inline V3<R> operator*(R s, const V3<R>& q) { return {s * q[0], s * q[1], s * q[2]}; }
template <class R> inline V3<R> operator-(const V3<R>& q) { return {-q[0], -q[1], -q[2]}; }
template <class R> inline V3<R>& operator+=(V3<R>& p, const V3<R>& q) { p[0] += q[0]; p[1] += q[1]; p[2] += q[2]; return p; }
template <class R> inline V3<R>& operator-=(V3<R>& p, const V3<R>& q) { p[0] -= q[0]; p[1] -= q[1]; p[2] -= q[2]; return p; }
// dot and norm in the order (x*x + y*y) + z*z, no fused multiply-add (the oracle is
// compiled with -ffp-contract=off).
template <class R> inline R dot(const V3<R>& p, const V3<R>& q) { return p[0] * q[0] + p[1] * q[1] + p[2] * q[2]; }
template <class R> inline R norm(const V3<R>& p) { return std::sqrt(dot(p, p)); }

template <class R> struct M3 {
    R a[3][3];
    M3() { for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) a[i][j] = R(0); }
    R* operator[](int i) { return a[i]; }
    const R* operator[](int i) const { return a[i]; }
};

// Cyclic Jacobi eigen-decomposition of a symmetric 3x3 matrix (the restatement of
// ti.sym_eig used at DSPH.py:684, spd_inverse.py:95, :150).  Returns eigenvalues in
// `ev` and eigenvectors as the COLUMNS of `Q`.  Fixed sweep cap, early exit when the
// off-diagonal mass falls below a relative threshold.
template <class R>
inline void sym_eig3(const M3<R>& Ain, R ev[3], M3<R>& Q) {
    R A[3][3];
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) A[i][j] = Ain[i][j];
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Q[i][j] = (i == j) ? R(1) : R(0);
    const R eps = sizeof(R) == 4 ? R(1e-14) : R(1e-30);
    for (int sweep = 0; sweep < 12; ++sweep) {
        R off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        R diag = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
        if (!(off > eps * diag) || off == R(0)) break;
        for (int p = 0; p < 2; ++p) {
            for (int q = p + 1; q < 3; ++q) {
                R apq = A[p][q];
                if (apq == R(0)) continue;
                R theta = (A[q][q] - A[p][p]) / (R(2) * apq);
                R t = (theta >= R(0) ? R(1) : R(-1)) / (std::fabs(theta) + std::sqrt(theta * theta + R(1)));
                R c = R(1) / std::sqrt(t * t + R(1));
                R s = t * c;
                R tau = s / (R(1) + c);
                A[p][p] -= t * apq;
                A[q][q] += t * apq;
                A[p][q] = A[q][p] = R(0);
                for (int r = 0; r < 3; ++r) {
                    if (r == p || r == q) continue;
                    R arp = A[r][p], arq = A[r][q];
                    A[r][p] = A[p][r] = arp - s * (arq + tau * arp);
                    A[r][q] = A[q][r] = arq + s * (arp - tau * arq);
                }
                for (int r = 0; r < 3; ++r) {
                    R qrp = Q[r][p], qrq = Q[r][q];
                    Q[r][p] = qrp - s * (qrq + tau * qrp);
                    Q[r][q] = qrq + s * (qrp - tau * qrq);
                }
            }
        }
    }
    for (int k = 0; k < 3; ++k) ev[k] = A[k][k];
}

// spd_inverse.py:45-50 -- per-eigendirection weight.
template <class R> inline R spd_weight(R e, R tol) {
    R u = std::min(R(1), std::max(R(0), (e - tol) / tol));
    R beta = u * u * (R(3) - R(2) * u);
    return beta / std::max(e, tol) + (R(1) - beta);
}

// spd_inverse.py:53-83
template <class R> inline void spd_inverse_2x2(R e00, R e01, R e10, R e11, R tol, R L[2][2]) {
    R a = e00, b = R(0.5) * (e01 + e10), d = e11;
    R disc = std::sqrt(std::max((a - d) * (a - d) + R(4) * b * b, R(0)));
    R e1 = R(0.5) * (a + d + disc);
    R e2 = R(0.5) * (a + d - disc);
    R n1x = 1, n1y = 0;
    R scale = std::fabs(a) + std::fabs(d) + R(1e-30);
    if (disc > R(1e-9) * scale) {
        R v1x = b, v1y = e1 - a, v2x = e1 - d, v2y = b;
        R l1 = std::sqrt(v1x * v1x + v1y * v1y), l2 = std::sqrt(v2x * v2x + v2y * v2y);
        if (l1 >= l2) { n1x = v1x / l1; n1y = v1y / l1; }
        else { n1x = v2x / l2; n1y = v2y / l2; }
    }
    R n2x = -n1y, n2y = n1x;
    R w1 = spd_weight(e1, tol), w2 = spd_weight(e2, tol);
    L[0][0] = w1 * (n1x * n1x) + w2 * (n2x * n2x);
    L[0][1] = w1 * (n1x * n1y) + w2 * (n2x * n2y);
    L[1][0] = w1 * (n1y * n1x) + w2 * (n2y * n2x);
    L[1][1] = w1 * (n1y * n1y) + w2 * (n2y * n2y);
}

// spd_inverse.py:129-157 (2x2 form of min_eig_vec)
template <class R> inline void min_eig_vec_2x2(R e00, R e01, R e10, R e11, R out[2]) {
    R a = e00, b = R(0.5) * (e01 + e10), d = e11;
    R disc = std::sqrt(std::max((a - d) * (a - d) + R(4) * b * b, R(0)));
    R e1 = R(0.5) * (a + d + disc);
    R n1x = 1, n1y = 0;
    R scale = std::fabs(a) + std::fabs(d) + R(1e-30);
    if (disc > R(1e-9) * scale) {
        R v1x = b, v1y = e1 - a, v2x = e1 - d, v2y = b;
        R l1 = std::sqrt(v1x * v1x + v1y * v1y), l2 = std::sqrt(v2x * v2x + v2y * v2y);
        if (l1 >= l2) { n1x = v1x / l1; n1y = v1y / l1; }
        else { n1x = v2x / l2; n1y = v2y / l2; }
    }
    out[0] = -n1y; out[1] = n1x;
}

// spd_inverse.py:86-101 -- the symmetrised matrix, its eigenpairs, the weighted sum.
template <class R> inline M3<R> spd_inverse_3x3(const M3<R>& E, R tol, R* min_eig = nullptr,
                                                R* min_vec = nullptr) {
    M3<R> Es;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Es[i][j] = R(0.5) * (E[i][j] + E[j][i]);
    R ev[3]; M3<R> Q;
    sym_eig3(Es, ev, Q);
    M3<R> L;
    for (int k = 0; k < 3; ++k) {
        R w = spd_weight(ev[k], tol);
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) L[i][j] += w * (Q[i][k] * Q[j][k]);
    }
    int kmin = 0;
    if (ev[1] < ev[kmin]) kmin = 1;
    if (ev[2] < ev[kmin]) kmin = 2;
    if (min_eig) *min_eig = std::min(ev[0], std::min(ev[1], ev[2]));
    if (min_vec) { min_vec[0] = Q[0][kmin]; min_vec[1] = Q[1][kmin]; min_vec[2] = Q[2][kmin]; }
    return L;
}

}  // namespace orc
