// ORACLE / TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library includes
// this file; it is used by the CPU oracle and by the harness that drives the
// reference's own CUDA kernels.
//
// FP64 restatements of the third-party arithmetic on the tracking path:
//   - Eigen Matrix<double,6,6>::ldlt().solve (Tracking/Tracking.cc:388).  Eigen
//     is not vendored with the reference (CMakeLists.txt:14 asks for >= 3.2);
//     this is a plain LDL^T factorisation with symmetric diagonal pivoting,
//     which returns the same solution up to rounding for the SPD systems the
//     tracker builds.
//   - Sophus::SE3d::exp (Tracking/Tracking.cc:389).  Sophus is not vendored.
//     Restated from the mathematics: tangent vector ordered (upsilon, omega);
//     R = Rodrigues(omega), t = V(omega) * upsilon with the left Jacobian
//     V = I + (1 - cos t)/t^2 W + (t - sin t)/t^3 W^2, Taylor series near 0.
//   - Eigen eulerAngles(0,1,2).array().sin().norm() (Tracking.cc:401): the
//     norm of the sines of an X-Y-Z Euler decomposition.  Any valid X-Y-Z
//     decomposition gives the same norm (the alternatives differ by pi shifts
//     that flip signs only), so a direct atan2/asin decomposition is used.
// Poses are 4x4 row-major double matrices, camera-to-world.
#ifndef FB_ORACLE_SE3_HPP
#define FB_ORACLE_SE3_HPP

#include <cmath>
#include <cstring>

namespace fbo {

inline void mat4_mul(const double* A, const double* B, double* C) {
    double T[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0;
            for (int k = 0; k < 4; ++k) s += A[i * 4 + k] * B[k * 4 + j];
            T[i * 4 + j] = s;
        }
    std::memcpy(C, T, sizeof T);
}

// Inverse of a rigid transform.
inline void mat4_rigid_inv(const double* A, double* B) {
    double T[16];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) T[i * 4 + j] = A[j * 4 + i];
    for (int i = 0; i < 3; ++i)
        T[i * 4 + 3] = -(T[i * 4 + 0] * A[3] + T[i * 4 + 1] * A[7] + T[i * 4 + 2] * A[11]);
    T[12] = T[13] = T[14] = 0;
    T[15] = 1;
    std::memcpy(B, T, sizeof T);
}

// General 4x4 inverse (Gauss-Jordan with partial pivoting); Eigen's
// Matrix4d::inverse() is used by the reference on matrices that are rigid up
// to rounding, for which this agrees with the rigid inverse to ~1e-16.
inline bool mat4_inv(const double* A, double* B) {
    double M[4][8];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 8; ++j) M[i][j] = j < 4 ? A[i * 4 + j] : (j - 4 == i ? 1.0 : 0.0);
    for (int c = 0; c < 4; ++c) {
        int p = c;
        for (int r = c + 1; r < 4; ++r)
            if (std::fabs(M[r][c]) > std::fabs(M[p][c])) p = r;
        if (M[p][c] == 0) return false;
        if (p != c)
            for (int j = 0; j < 8; ++j) std::swap(M[p][j], M[c][j]);
        double inv = 1.0 / M[c][c];
        for (int j = 0; j < 8; ++j) M[c][j] *= inv;
        for (int r = 0; r < 4; ++r)
            if (r != c) {
                double f = M[r][c];
                if (f != 0)
                    for (int j = 0; j < 8; ++j) M[r][j] -= f * M[c][j];
            }
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) B[i * 4 + j] = M[i][j + 4];
    return true;
}

// Solve A x = b for symmetric A (n <= 6) by LDL^T with symmetric pivoting.
// Returns false when a pivot is exactly zero (the solution is then NaN).
inline bool ldlt_solve(const double* Ain, const double* bin, double* x, int n = 6) {
    double A[36], b[6];
    int perm[6];
    std::memcpy(A, Ain, sizeof(double) * n * n);
    std::memcpy(b, bin, sizeof(double) * n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    double L[36] = {0}, D[6] = {0};
    for (int k = 0; k < n; ++k) {
        // pivot: the largest remaining diagonal entry
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(A[i * n + i]) > std::fabs(A[p * n + p])) p = i;
        if (p != k) {
            for (int j = 0; j < n; ++j) std::swap(A[k * n + j], A[p * n + j]);
            for (int i = 0; i < n; ++i) std::swap(A[i * n + k], A[i * n + p]);
            for (int j = 0; j < k; ++j) std::swap(L[k * n + j], L[p * n + j]);
            std::swap(perm[k], perm[p]);
        }
        double d = A[k * n + k];
        for (int j = 0; j < k; ++j) d -= L[k * n + j] * L[k * n + j] * D[j];
        D[k] = d;
        L[k * n + k] = 1;
        for (int i = k + 1; i < n; ++i) {
            double s = A[i * n + k];
            for (int j = 0; j < k; ++j) s -= L[i * n + j] * L[k * n + j] * D[j];
            L[i * n + k] = d != 0 ? s / d : NAN;
        }
    }
    // solve P^T L D L^T P x = b
    double y[6];
    for (int i = 0; i < n; ++i) {
        double s = b[perm[i]];
        for (int j = 0; j < i; ++j) s -= L[i * n + j] * y[j];
        y[i] = s;
    }
    for (int i = 0; i < n; ++i) y[i] /= D[i];
    double z[6];
    for (int i = n - 1; i >= 0; --i) {
        double s = y[i];
        for (int j = i + 1; j < n; ++j) s -= L[j * n + i] * z[j];
        z[i] = s;
    }
    for (int i = 0; i < n; ++i) x[perm[i]] = z[i];
    for (int i = 0; i < n; ++i)
        if (D[i] == 0) return false;
    return true;
}

// The same solve without pivoting, in the operation order of the library's
// device solver (the normal matrix is symmetric positive definite, so no
// pivot is needed): D and L column by column with L = t * (1 / d), forward
// substitution, scaling by 1 / D, back substitution.  Used to compare the
// library's tracker bit for bit.
inline void ldlt_solve_nopivot(const double* A, const double* b, double* x) {
    double L[6][6] = {}, D[6], Dinv[6], y[6];
    for (int k = 0; k < 6; ++k) {
        double d = A[k * 6 + k];
        for (int j = 0; j < k; ++j) d -= L[k][j] * L[k][j] * D[j];
        D[k] = d;
        const double inv = 1.0 / d;
        Dinv[k] = inv;
        for (int i = k + 1; i < 6; ++i) {
            double t = A[i * 6 + k];
            for (int j = 0; j < k; ++j) t -= L[i][j] * L[k][j] * D[j];
            L[i][k] = t * inv;
        }
    }
    for (int i = 0; i < 6; ++i) {
        double t = b[i];
        for (int j = 0; j < i; ++j) t -= L[i][j] * y[j];
        y[i] = t;
    }
    for (int i = 0; i < 6; ++i) y[i] *= Dinv[i];
    for (int i = 5; i >= 0; --i) {
        double t = y[i];
        for (int j = i + 1; j < 6; ++j) t -= L[j][i] * x[j];
        x[i] = t;
    }
}

// exp of the se(3) tangent (upsilon[3], omega[3]) into a 4x4 row-major matrix.
inline void se3_exp(const double* xi, double* T) {
    const double* u = xi;
    const double* w = xi + 3;
    double th2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    double th = std::sqrt(th2);
    double W[9] = {0, -w[2], w[1], w[2], 0, -w[0], -w[1], w[0], 0};
    double W2[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += W[i * 3 + k] * W[k * 3 + j];
            W2[i * 3 + j] = s;
        }
    double a, b, c;  // R = I + a W + b W^2 ; V = I + b W + c W^2
    if (th < 1e-5) {
        a = 1 - th2 / 6 + th2 * th2 / 120;
        b = 0.5 - th2 / 24 + th2 * th2 / 720;
        c = 1.0 / 6 - th2 / 120 + th2 * th2 / 5040;
    } else {
        a = std::sin(th) / th;
        b = (1 - std::cos(th)) / th2;
        c = (th - std::sin(th)) / (th2 * th);
    }
    double R[9], V[9];
    for (int i = 0; i < 9; ++i) {
        double I = (i % 4 == 0) ? 1.0 : 0.0;
        R[i] = I + a * W[i] + b * W2[i];
        V[i] = I + b * W[i] + c * W2[i];
    }
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) T[i * 4 + j] = R[i * 3 + j];
        T[i * 4 + 3] = V[i * 3 + 0] * u[0] + V[i * 3 + 1] * u[1] + V[i * 3 + 2] * u[2];
    }
    T[12] = T[13] = T[14] = 0;
    T[15] = 1;
}

// || sin(eulerAngles(0,1,2)) || of the rotation block of a 4x4 matrix.
inline double euler_sin_norm(const double* T) {
    double r00 = T[0], r01 = T[1], r02 = T[2], r12 = T[6], r22 = T[10];
    double a = std::atan2(-r12, r22);
    double b = std::atan2(r02, std::sqrt(r00 * r00 + r01 * r01));
    double c = std::atan2(-r01, r00);
    double sa = std::sin(a), sb = std::sin(b), sc = std::sin(c);
    return std::sqrt(sa * sa + sb * sb + sc * sc);
}

// Unpack 29 reduction sums (28 upper-triangle products of a 7-vector row and
// a count) into a symmetric 6x6 A (row-major) and b, as CreateMatrix<6,7>
// does (Tracking/Reduction.cu:6-16).
template <typename F>
inline void unpack_29(const F* s, double* A, double* b) {
    int shift = 0;
    for (int i = 0; i < 6; ++i)
        for (int j = i; j < 7; ++j) {
            double v = (double)s[shift++];
            if (j == 6)
                b[i] = v;
            else
                A[j * 6 + i] = A[i * 6 + j] = v;
        }
}

}  // namespace fbo

#endif
