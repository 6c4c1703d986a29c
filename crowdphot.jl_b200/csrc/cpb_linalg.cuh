// cpb_linalg.cuh -- small dense linear algebra shared by the device fitters.
//
//   sym_givens        Givens rotation of Krylov.jl's LSQR (Paige & Saunders 1982)
//   chol_inv_small    cholesky!(Symmetric(A)) then F \ I  (levenberg_marquardt.jl:366-388)
//   pinv_small        the pinv fallback of covariance!  (levenberg_marquardt.jl:366-388)
#pragma once

#include <cuda_runtime.h>

namespace cpb {

constexpr double kLinEps64 = 2.220446049250313e-16;

__device__ __forceinline__ double sgn(double v) { return v > 0 ? 1.0 : (v < 0 ? -1.0 : 0.0); }
__device__ __forceinline__ void sym_givens(double a, double b, double& c, double& s, double& rho) {
    if (b == 0) {
        c = (a == 0) ? 1.0 : sgn(a);
        s = 0;
        rho = fabs(a);
    } else if (a == 0) {
        c = 0;
        s = sgn(b);
        rho = fabs(b);
    } else if (fabs(b) > fabs(a)) {
        double t = a / b;
        s = sgn(b) / sqrt(1.0 + t * t);
        c = s * t;
        rho = b / s;
    } else {
        double t = b / a;
        c = sgn(a) / sqrt(1.0 + t * t);
        s = c * t;
        rho = a / c;
    }
}

// Per-star p x p covariance from the Gram block (:1305-1329,
// levenberg_marquardt.jl:366-388): ridge 1e-12 tr, Cholesky inverse,
// Jacobi pseudo-inverse fallback, reweighted scaling by cost/dof.
__device__ inline void pinv_small(double* A, int n, double* inv) {
    double V[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) {
            double s = 0.5 * (A[i + j * n] + A[j + i * n]);
            A[i + j * n] = A[j + i * n] = s;
        }
    for (int i = 0; i < 9; ++i) V[i] = 0;
    for (int i = 0; i < n; ++i) V[i + i * n] = 1;
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0;
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) off += A[i + j * n] * A[i + j * n];
        if (off < 1e-300) break;
        for (int pp = 0; pp < n; ++pp)
            for (int q = pp + 1; q < n; ++q) {
                double apq = A[pp + q * n];
                if (apq == 0) continue;
                double tau = (A[q + q * n] - A[pp + pp * n]) / (2 * apq);
                double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1 + tau * tau));
                double c = 1 / sqrt(1 + t * t), s = t * c;
                for (int k = 0; k < n; ++k) {
                    double akp = A[k + pp * n], akq = A[k + q * n];
                    A[k + pp * n] = c * akp - s * akq;
                    A[k + q * n] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    double apk = A[pp + k * n], aqk = A[q + k * n];
                    A[pp + k * n] = c * apk - s * aqk;
                    A[q + k * n] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    double vkp = V[k + pp * n], vkq = V[k + q * n];
                    V[k + pp * n] = c * vkp - s * vkq;
                    V[k + q * n] = s * vkp + c * vkq;
                }
            }
    }
    double smax = 0;
    for (int i = 0; i < n; ++i) smax = fmax(smax, fabs(A[i + i * n]));
    double tol = kLinEps64 * n * smax;
    for (int i = 0; i < n * n; ++i) inv[i] = 0;
    for (int e = 0; e < n; ++e) {
        double lam = A[e + e * n];
        if (!(fabs(lam) > tol)) continue;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) inv[i + j * n] += V[i + e * n] * V[j + e * n] / lam;
    }
}

__device__ inline bool chol_inv_small(const double* A, int n, double* inv) {
    double U[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = 0; j < n; ++j)
        for (int i = 0; i <= j; ++i) {
            double s = A[i + j * n];
            for (int k = 0; k < i; ++k) s -= U[k + i * n] * U[k + j * n];
            if (i == j) {
                if (!(s > 0)) return false;
                U[j + j * n] = sqrt(s);
            } else {
                U[i + j * n] = s / U[i + i * n];
            }
        }
    for (int c = 0; c < n; ++c) {
        double y[3], xx[3];
        for (int i = 0; i < n; ++i) {
            double s = (i == c) ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) s -= U[k + i * n] * y[k];
            y[i] = s / U[i + i * n];
        }
        for (int i = n - 1; i >= 0; --i) {
            double s = y[i];
            for (int k = i + 1; k < n; ++k) s -= U[i + k * n] * xx[k];
            xx[i] = s / U[i + i * n];
        }
        for (int i = 0; i < n; ++i) inv[i + c * n] = xx[i];
    }
    return true;
}

}  // namespace cpb
