// oracle_lsqr.cpp -- TEST INFRASTRUCTURE ONLY (the oracle): damped LSQR.
// Scope, provenance and parity status are stated in oracle_lsqr.hpp.
#include "oracle_lsqr.hpp"

#include <algorithm>
#include <limits>

namespace orc {

LsqrStats lsqr(int64_t m, int64_t n, const std::function<void(const double*, double*)>& Av,
               const std::function<void(const double*, double*)>& Atu, const double* b, double lambda,
               int itmax, double atol, double btol, double* x) {
    const double eps = std::numeric_limits<double>::epsilon();
    const double axtol = std::sqrt(eps), etol = std::sqrt(eps), conlim = 1.0 / std::sqrt(eps);
    const double ctol = conlim > 0 ? 1.0 / conlim : 0.0, rtol = 0.0;
    const int window = 5;
    LsqrStats st;
    std::fill(x, x + n, 0.0);
    std::vector<double> u(b, b + m), v(n), w(n), tmpm(m), tmpn(n);
    double beta1 = 0;
    for (int64_t i = 0; i < m; ++i) beta1 += u[i] * u[i];
    beta1 = std::sqrt(beta1);
    if (beta1 == 0) {
        st.status = 4;
        return st;
    }
    double beta = beta1;
    for (auto& e : u) e *= 1.0 / beta1;
    Atu(u.data(), v.data());
    double Anorm2 = 0;
    for (int64_t i = 0; i < n; ++i) Anorm2 += v[i] * v[i];
    double Anorm = std::sqrt(Anorm2);
    double alpha = Anorm;
    double dNorm2 = 0, xNorm = 0, xNorm2 = 0, c2 = -1, s2 = 0, z = 0, xENorm2 = 0, err_lbnd = 0;
    double err_vec[window] = {0, 0, 0, 0, 0};
    double rNorm = beta1, res2 = 0;
    double ArNorm = alpha * beta, ArNorm0 = ArNorm;
    if (alpha == 0) {
        st.status = 4;
        return st;
    }
    for (auto& e : v) e *= 1.0 / alpha;
    w = v;
    double phibar = beta1, rhobar = alpha;
    bool solved = (ArNorm / (Anorm * rNorm) <= axtol) || (1.0 + ArNorm / (Anorm * rNorm) <= 1.0);
    bool zero_resid = (rNorm / beta1 <= axtol) || (1.0 + rNorm / beta1 <= 1.0);
    (void)zero_resid;
    bool ill_cond = false, tired = (0 >= itmax), fwd_err = false;
    int iter = 0;
    const double lam2 = lambda * lambda;
    while (!(solved || tired || ill_cond)) {
        ++iter;
        // beta_{k+1} u_{k+1} = A v_k - alpha_k u_k
        Av(v.data(), tmpm.data());
        for (int64_t i = 0; i < m; ++i) u[i] = tmpm[i] - alpha * u[i];
        beta = 0;
        for (int64_t i = 0; i < m; ++i) beta += u[i] * u[i];
        beta = std::sqrt(beta);
        if (beta != 0) {
            for (auto& e : u) e *= 1.0 / beta;
            Anorm2 = Anorm2 + alpha * alpha + beta * beta;
            if (lambda > 0) Anorm2 += lam2;
            // alpha_{k+1} v_{k+1} = A' u_{k+1} - beta_{k+1} v_k
            Atu(u.data(), tmpn.data());
            for (int64_t i = 0; i < n; ++i) v[i] = tmpn[i] - beta * v[i];
            alpha = 0;
            for (int64_t i = 0; i < n; ++i) alpha += v[i] * v[i];
            alpha = std::sqrt(alpha);
            if (alpha != 0)
                for (auto& e : v) e *= 1.0 / alpha;
        }
        // eliminate the damping parameter
        double c1, s1, rhobar1;
        sym_givens(rhobar, lambda, c1, s1, rhobar1);
        double psi = s1 * phibar;
        phibar = c1 * phibar;
        // eliminate beta
        double c, s, rho;
        sym_givens(rhobar1, beta, c, s, rho);
        double phi = c * phibar;
        phibar = s * phibar;
        xENorm2 = xENorm2 + phi * phi;
        err_vec[iter % window] = phi;
        if (iter >= window) {
            double e2 = 0;
            for (int k = 0; k < window; ++k) e2 += err_vec[k] * err_vec[k];
            err_lbnd = std::sqrt(e2);
        }
        double tau = s * phi;
        double theta = s * alpha;
        rhobar = -c * alpha;
        double ww = 0;
        for (int64_t i = 0; i < n; ++i) ww += w[i] * w[i];
        dNorm2 += ww / (rho * rho);
        double sigma = phi / rho;
        for (int64_t i = 0; i < n; ++i) x[i] += sigma * w[i];
        double tr = -theta / rho;
        for (int64_t i = 0; i < n; ++i) w[i] = v[i] + tr * w[i];
        // estimate ||x|| with a rotation on the right
        double delta = s2 * rho;
        double gambar = -c2 * rho;
        double rhs = phi - delta * z;
        double zbar = rhs / gambar;
        xNorm = std::sqrt(xNorm2 + zbar * zbar);
        double gamma;
        sym_givens(gambar, theta, c2, s2, gamma);
        z = rhs / gamma;
        xNorm2 += z * z;
        Anorm = std::sqrt(Anorm2);
        double Acond = Anorm * std::sqrt(dNorm2);
        double res1 = phibar * phibar;
        res2 += psi * psi;
        rNorm = std::sqrt(res1 + res2);
        ArNorm = alpha * std::fabs(tau);
        double test1 = rNorm / beta1;
        double test2 = ArNorm / (Anorm * rNorm);
        double test3 = 1.0 / Acond;
        double t1 = test1 / (1.0 + Anorm * xNorm / beta1);
        double rNormtol = btol + axtol * Anorm * xNorm / beta1;
        bool ill_cond_mach = (1.0 + test3 <= 1.0);
        bool solved_mach = (1.0 + test2 <= 1.0);
        bool zero_resid_mach = (1.0 + t1 <= 1.0);
        tired = iter >= itmax;
        bool ill_cond_lim = (test3 <= ctol);
        bool solved_lim = (test2 <= axtol);
        bool solved_opt = ArNorm <= atol + rtol * ArNorm0;
        bool zero_resid_lim = (test1 <= rNormtol);
        if (iter >= window) fwd_err = err_lbnd <= etol * std::sqrt(xENorm2);
        ill_cond = ill_cond_mach || ill_cond_lim;
        bool zr = zero_resid_mach || zero_resid_lim;
        solved = solved_mach || solved_lim || solved_opt || zr || fwd_err;
        if (solved) st.status = zr ? 2 : 1;
        else if (ill_cond) st.status = 3;
    }
    st.iters = iter;
    return st;
}

LsqrStats lsmr(int64_t m, int64_t n, const std::function<void(const double*, double*)>& Av,
               const std::function<void(const double*, double*)>& Atu, const double* b, double lambda,
               int itmax, double atol, double btol, double* x) {
    const double eps = std::numeric_limits<double>::epsilon();
    const double axtol = std::sqrt(eps), conlim = 1.0 / std::sqrt(eps);
    const double ctol = conlim > 0 ? 1.0 / conlim : 0.0, rtol = 0.0;
    LsqrStats st;
    std::fill(x, x + n, 0.0);
    std::vector<double> u(b, b + m), v(n), h(n), hbar(n, 0.0), tmpm(m), tmpn(n);
    double beta1 = 0;
    for (int64_t i = 0; i < m; ++i) beta1 += u[i] * u[i];
    beta1 = std::sqrt(beta1);
    if (beta1 == 0) {
        st.status = 4;
        return st;
    }
    double beta = beta1;
    for (auto& e : u) e *= 1.0 / beta1;
    Atu(u.data(), v.data());
    double alpha = 0;
    for (int64_t i = 0; i < n; ++i) alpha += v[i] * v[i];
    alpha = std::sqrt(alpha);
    if (alpha == 0) {
        st.status = 4;
        return st;
    }
    for (auto& e : v) e *= 1.0 / alpha;
    // QR factorisation state (Fong & Saunders, section 2)
    double zetabar = alpha * beta, alphabar = alpha, rho = 1, rhobar = 1, cbar = 1, sbar = 0, zeta = 0;
    h = v;
    // ||r|| estimate state (section 3.4)
    double betadd = beta, betad = 0, rhodold = 1, tautildeold = 0, thetatilde = 0, d = 0;
    // ||A||, cond(A) estimates (section 4)
    double Anorm2 = alpha * alpha, maxrbar = 0, minrbar = 1e100;
    const double ArNorm0 = alpha * beta;
    bool solved = false, tired = (0 >= itmax), ill_cond = false;
    int iter = 0;
    while (!(solved || tired || ill_cond)) {
        ++iter;
        // Golub-Kahan step, as in lsqr
        Av(v.data(), tmpm.data());
        for (int64_t i = 0; i < m; ++i) u[i] = tmpm[i] - alpha * u[i];
        beta = 0;
        for (int64_t i = 0; i < m; ++i) beta += u[i] * u[i];
        beta = std::sqrt(beta);
        if (beta != 0) {
            for (auto& e : u) e *= 1.0 / beta;
            Atu(u.data(), tmpn.data());
            for (int64_t i = 0; i < n; ++i) v[i] = tmpn[i] - beta * v[i];
            alpha = 0;
            for (int64_t i = 0; i < n; ++i) alpha += v[i] * v[i];
            alpha = std::sqrt(alpha);
            if (alpha != 0)
                for (auto& e : v) e *= 1.0 / alpha;
        }
        // rotation eliminating the damping, then the one turning B into R
        double chat, shat, alphahat;
        sym_givens(alphabar, lambda, chat, shat, alphahat);
        const double rhoold = rho;
        double c, s;
        sym_givens(alphahat, beta, c, s, rho);
        const double thetanew = s * alpha;
        alphabar = c * alpha;
        // rotation turning R' into Rbar
        const double rhobarold = rhobar, zetaold = zeta;
        const double thetabar = sbar * rho, rhotemp = cbar * rho;
        sym_givens(cbar * rho, thetanew, cbar, sbar, rhobar);
        zeta = cbar * zetabar;
        zetabar = -sbar * zetabar;
        // h, hbar, x
        const double kh = thetabar * rho / (rhoold * rhobarold);
        const double kx = zeta / (rho * rhobar);
        const double kv = thetanew / rho;
        double xx = 0;
        for (int64_t i = 0; i < n; ++i) {
            hbar[i] = h[i] - kh * hbar[i];
            x[i] += kx * hbar[i];
            h[i] = v[i] - kv * h[i];
            xx += x[i] * x[i];
        }
        // ||r|| estimate
        const double betaacute = chat * betadd, betacheck = -shat * betadd;
        const double betahat = c * betaacute;
        betadd = -s * betaacute;
        const double thetatildeold = thetatilde;
        double ctildeold, stildeold, rhotildeold;
        sym_givens(rhodold, thetabar, ctildeold, stildeold, rhotildeold);
        thetatilde = stildeold * rhobar;
        rhodold = ctildeold * rhobar;
        betad = -stildeold * betad + ctildeold * betahat;
        tautildeold = (zetaold - thetatildeold * tautildeold) / rhotildeold;
        const double taud = (zeta - thetatilde * tautildeold) / rhodold;
        d += betacheck * betacheck;
        const double rNorm = std::sqrt(d + (betad - taud) * (betad - taud) + betadd * betadd);
        // ||A|| and cond(A)
        Anorm2 += beta * beta;
        const double Anorm = std::sqrt(Anorm2);
        Anorm2 += alpha * alpha;
        maxrbar = std::max(maxrbar, rhobarold);
        if (iter > 1) minrbar = std::min(minrbar, rhobarold);
        const double Acond = std::max(maxrbar, rhotemp) / std::min(minrbar, rhotemp);
        // stopping tests
        const double ArNorm = std::fabs(zetabar);
        const double xNorm = std::sqrt(xx);
        const double test1 = rNorm / beta1;
        const double test2 = ArNorm / (Anorm * rNorm);
        const double test3 = 1.0 / Acond;
        const double t1 = test1 / (1.0 + Anorm * xNorm / beta1);
        const double rNormtol = btol + axtol * Anorm * xNorm / beta1;
        tired = iter >= itmax;
        ill_cond = (1.0 + test3 <= 1.0) || (test3 <= ctol);
        const bool zr = (1.0 + t1 <= 1.0) || (test1 <= rNormtol);
        solved = (1.0 + test2 <= 1.0) || (test2 <= axtol) || (ArNorm <= atol + rtol * ArNorm0) || zr;
        if (solved) st.status = zr ? 2 : 1;
        else if (ill_cond) st.status = 3;
    }
    st.iters = iter;
    return st;
}

}  // namespace orc
